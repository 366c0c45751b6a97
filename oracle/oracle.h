/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 * Groth16-level restatement of the reference CPU prover, plus a flat
 * byte-buffer API (oracle_*) that the Python tests bind through ctypes.
 */
#ifndef G16_ORACLE_H
#define G16_ORACLE_H
#include "bn254.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int log_n;
    size_t n;
    fp_t omega, omega_inv, n_inv, shift;
    fp_t *tw, *tw_inv;   /* omega^i, omega^-i for i < n/2 */
    fp_t *coset;         /* shift^bitrev(p) / n, p < n */
} domain_t;

int  domain_root(int log_n, fp_t *out);
int  domain_init(domain_t *d, int log_n);
void domain_free(domain_t *d);
void bitrev_permute(fp_t *a, size_t n);
void ntt_forward(const domain_t *d, fp_t *a);
void ntt_inverse(const domain_t *d, fp_t *a);
void intt_coset_ntt(const domain_t *d, fp_t *a);
void distribute_powers(fp_t *a, size_t n, const fp_t *shift);

int  msm_window_size(size_t m);
/* scalars in standard form; infinity bases contribute nothing */
void msm_g1(g1j_t *out, const g1a_t *bases, const fp_t *scalars_std, size_t n);
void msm_g2(g2j_t *out, const g2a_t *bases, const fp_t *scalars_std, size_t n);

typedef struct {
    uint32_t n_vars, n_public, domain_size;
    g1a_t alpha_g1, beta_g1, delta_g1;
    g2a_t beta_g2, gamma_g2, delta_g2;
    g1a_t *ic;
    size_t n_ic;
    uint32_t *row_ptr[2];   /* CSR by constraint, domain_size + 1 entries */
    uint32_t *signal[2];
    fp_t *coef[2];          /* Montgomery form */
    size_t nnz[2];
    g1a_t *a_query, *b_g1_query, *l_query, *h_query;
    g2a_t *b_g2_query;
    int h_basis;            /* 0 snarkjs odd coset (n_h = domain_size), 1 gnark bit-reversed (n_h = domain_size - 1) */
    size_t n_h;             /* H bases */
} zkey_t;

int  zkey_parse(zkey_t *k, const uint8_t *bytes, size_t len, char *err, size_t errlen);
void zkey_free(zkey_t *k);

typedef struct { g1a_t a; g2a_t b; g1a_t c; } proof_t;
typedef struct { g1j_t a_g1; g2j_t b_g2; g1j_t b_g1, l_g1, h_g1; } msm_outputs_t;

/* witness in Montgomery form (the reference's &[Fr]), length n_vars */
int  groth16_compute_h(const zkey_t *k, const fp_t *w, fp_t *h /* domain_size, Montgomery */);
void groth16_gather(const zkey_t *k, const fp_t *w, fp_t *a, fp_t *b /* domain_size rows each */);
int  groth16_compute_h_from_rows(const zkey_t *k, const fp_t *a_rows, const fp_t *b_rows, size_t n_rows, fp_t *h);
int  groth16_msms(const zkey_t *k, const fp_t *w, const fp_t *h, msm_outputs_t *out);
void groth16_assemble(const zkey_t *k, const msm_outputs_t *m, const fp_t *r, const fp_t *s, proof_t *p);
int  groth16_prove(const zkey_t *k, const fp_t *w, const fp_t *r, const fp_t *s, proof_t *p);
/* stages 1-11 from A.w and B.w rows (h_and_msms_from_rows, cpu.rs:384-471), either H basis */
int  groth16_prove_rows(const zkey_t *k, const fp_t *w, const fp_t *a_rows, const fp_t *b_rows, size_t n_rows,
                        const fp_t *r, const fp_t *s, proof_t *p);

/* gnark v0.14 proving-key dump + verifying key -> key with the gnark H basis (gnark.c) */
int  gnark_parse(zkey_t *k, const uint8_t *pk, size_t pk_len, const uint8_t *vk, size_t vk_len, char *err,
                 size_t errlen);
/* coset values of H -> gnark's bit-reversed coefficients; -1 if coefficient n-1 is not zero */
int  groth16_gnark_coefficients(const zkey_t *k, fp_t *h);
int  groth16_verify(const g1a_t *alpha, const g2a_t *beta, const g2a_t *gamma, const g2a_t *delta,
                    const g1a_t *ic, size_t n_ic, const fp_t *pub_mont, const proof_t *p);

/* packed point codecs: Montgomery LE coordinates, infinity = all-zero bytes */
void pack_g1(uint8_t *out64, const g1a_t *p);
int  unpack_g1(g1a_t *p, const uint8_t *in64);     /* 0 on non-canonical coordinate */
void pack_g2(uint8_t *out128, const g2a_t *p);
int  unpack_g2(g2a_t *p, const uint8_t *in128);

#ifdef __cplusplus
}
#endif
#endif
