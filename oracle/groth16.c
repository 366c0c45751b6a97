/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Stages 0-11 of the reference CPU prover and its verifier:
 *   - stage 0, CpuCircuit::gather (crates/groth16/src/cpu.rs:140-174):
 *     A[c] = sum over CSR row c of coef * w[signal], same for B, C = A*B
 *     (cpu.rs:316-341); or the caller's rows, zero padded, with C = A*B
 *     (h_and_msms_from_rows, cpu.rs:384-425);
 *   - stages 1-4, coset_h (cpu.rs:191-252): intt_coset_ntt on A, B and C,
 *     then H = A*B - C with no division by Z (cpu.rs:230-246);
 *   - stages 5-9, msms_with (cpu.rs:477-632): A over a_query, B over
 *     b_g2_query and b_g1_query, L over l_query with w[n_public+1..], H over
 *     h_query, all scalars in standard form;
 *   - stage 11, BlinderTerms::new + assemble_from_terms
 *     (crates/groth16/src/prove.rs:335-346, 391-430);
 *   - verify_unchecked + check_proof (crates/groth16/src/verify.rs:49-137):
 *     e(-A,B) e(alpha,beta) e(Lbar,gamma) e(C,delta) == 1.
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>

#define R (&FR)

/* stage 0: A.w and B.w, one row per domain row (CpuCircuit::gather, cpu.rs:140-174) */
void groth16_gather(const zkey_t *k, const fp_t *w, fp_t *a, fp_t *b) {
    size_t n = k->domain_size;
    fp_t *ab[2] = {a, b};
    for (int m = 0; m < 2; m++) {
        fp_t *out = ab[m];
#pragma omp parallel for schedule(static)
        for (long row = 0; row < (long)n; row++) {
            fp_t acc = {{0}};
            for (uint32_t t = k->row_ptr[m][row]; t < k->row_ptr[m][row + 1]; t++) {
                fp_t prod;
                fp_mul(R, &prod, &k->coef[m][t], &w[k->signal[m][t]]);
                fp_add(R, &acc, &acc, &prod);
            }
            out[row] = acc;
        }
    }
}

/* stages 1-4 from the rows (h_and_msms_from_rows, cpu.rs:384-425): rows past
 * n_rows are zero, C = A*B */
int groth16_compute_h_from_rows(const zkey_t *k, const fp_t *a_rows, const fp_t *b_rows, size_t n_rows, fp_t *h) {
    size_t n = k->domain_size;
    if (n_rows > n) return -1;
    int log_n = 0;
    while (((size_t)1 << log_n) < n) log_n++;
    domain_t d;
    if (domain_init(&d, log_n) != 0) return -1;
    fp_t *b = calloc(n, sizeof(fp_t));
    fp_t *c = malloc(n * sizeof(fp_t));
    memset(h, 0, n * sizeof(fp_t));
    memcpy(h, a_rows, n_rows * sizeof(fp_t));
    memcpy(b, b_rows, n_rows * sizeof(fp_t));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) fp_mul(R, &c[i], &h[i], &b[i]);
    intt_coset_ntt(&d, h);
    intt_coset_ntt(&d, b);
    intt_coset_ntt(&d, c);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        fp_t t;
        fp_mul(R, &t, &h[i], &b[i]);
        fp_sub(R, &h[i], &t, &c[i]);
    }
    free(b);
    free(c);
    domain_free(&d);
    return 0;
}

int groth16_compute_h(const zkey_t *k, const fp_t *w, fp_t *h) {
    size_t n = k->domain_size;
    int log_n = 0;
    while (((size_t)1 << log_n) < n) log_n++;
    domain_t d;
    if (domain_init(&d, log_n) != 0) return -1;
    fp_t *ab[2];
    ab[0] = h;
    ab[1] = malloc(n * sizeof(fp_t));
    fp_t *c = malloc(n * sizeof(fp_t));
    groth16_gather(k, w, ab[0], ab[1]);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) fp_mul(R, &c[i], &ab[0][i], &ab[1][i]);
    intt_coset_ntt(&d, ab[0]);
    intt_coset_ntt(&d, ab[1]);
    intt_coset_ntt(&d, c);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; i++) {
        fp_t t;
        fp_mul(R, &t, &ab[0][i], &ab[1][i]);
        fp_sub(R, &h[i], &t, &c[i]);
    }
    free(ab[1]);
    free(c);
    domain_free(&d);
    return 0;
}

int groth16_msms(const zkey_t *k, const fp_t *w, const fp_t *h, msm_outputs_t *out) {
    size_t nv = k->n_vars, n = k->n_h ? k->n_h : k->domain_size;
    fp_t *ws = malloc(nv * sizeof(fp_t)), *hs = malloc(n * sizeof(fp_t));
    for (size_t i = 0; i < nv; i++) fp_from_mont(R, &ws[i], &w[i]);
    for (size_t i = 0; i < n; i++) fp_from_mont(R, &hs[i], &h[i]);
    size_t off = (size_t)k->n_public + 1;
    msm_g1(&out->a_g1, k->a_query, ws, nv);
    msm_g2(&out->b_g2, k->b_g2_query, ws, nv);
    msm_g1(&out->b_g1, k->b_g1_query, ws, nv);
    msm_g1(&out->l_g1, k->l_query, ws + off, nv - off);
    msm_g1(&out->h_g1, k->h_query, hs, n);
    free(ws);
    free(hs);
    return 0;
}

static void g1_mul_fr(g1j_t *r, const g1a_t *p, const fp_t *k_mont) {
    fp_t k;
    fp_from_mont(R, &k, k_mont);
    g1j_t pj;
    g1j_from_affine(&pj, p);
    g1j_mul(r, &pj, &k);
}

void groth16_assemble(const zkey_t *k, const msm_outputs_t *m, const fp_t *r, const fp_t *s, proof_t *p) {
    g1j_t d1r, d1s, d1rs, t, pi_a, pib1, pi_c, as, b1r;
    g2j_t d2s, pi_b, t2;
    fp_t rs;
    fp_mul(R, &rs, r, s);
    g1_mul_fr(&d1r, &k->delta_g1, r);
    g1_mul_fr(&d1s, &k->delta_g1, s);
    g1_mul_fr(&d1rs, &k->delta_g1, &rs);
    fp_t s_std;
    fp_from_mont(R, &s_std, s);
    g2j_from_affine(&t2, &k->delta_g2);
    g2j_mul(&d2s, &t2, &s_std);

    /* pi_a = a + alpha + r delta1 */
    g1j_add_affine(&pi_a, &m->a_g1, &k->alpha_g1);
    g1j_add(&pi_a, &pi_a, &d1r);
    /* pi_b = b2 + beta2 + s delta2 */
    g2j_add_affine(&pi_b, &m->b_g2, &k->beta_g2);
    g2j_add(&pi_b, &pi_b, &d2s);
    /* pib1 = b1 + beta1 + s delta1 */
    g1j_add_affine(&pib1, &m->b_g1, &k->beta_g1);
    g1j_add(&pib1, &pib1, &d1s);
    /* pi_c = l + h + s pi_a + r pib1 - rs delta1 */
    fp_t r_std;
    fp_from_mont(R, &r_std, r);
    g1j_mul(&as, &pi_a, &s_std);
    g1j_mul(&b1r, &pib1, &r_std);
    g1j_add(&pi_c, &m->l_g1, &m->h_g1);
    g1j_add(&pi_c, &pi_c, &as);
    g1j_add(&pi_c, &pi_c, &b1r);
    g1j_neg(&t, &d1rs);
    g1j_add(&pi_c, &pi_c, &t);

    g1j_to_affine(&p->a, &pi_a);
    g2j_to_affine(&p->b, &pi_b);
    g1j_to_affine(&p->c, &pi_c);
}

int groth16_prove(const zkey_t *k, const fp_t *w, const fp_t *r, const fp_t *s, proof_t *p) {
    fp_t *h = malloc((size_t)k->domain_size * sizeof(fp_t));
    if (groth16_compute_h(k, w, h) != 0) { free(h); return -1; }
    msm_outputs_t m;
    groth16_msms(k, w, h, &m);
    free(h);
    groth16_assemble(k, &m, r, s, p);
    return 0;
}

/* stages 1-11 from the caller's rows (h_and_msms_from_rows, cpu.rs:384-471): for a
 * gnark key H goes to its bit-reversed coefficients, the MSM runs over the n - 1
 * Z bases, and its result is multiplied by -1/2, which is 1/t on the odd coset */
int groth16_prove_rows(const zkey_t *k, const fp_t *w, const fp_t *a_rows, const fp_t *b_rows, size_t n_rows,
                       const fp_t *r, const fp_t *s, proof_t *p) {
    fp_t *h = malloc((size_t)k->domain_size * sizeof(fp_t));
    if (groth16_compute_h_from_rows(k, a_rows, b_rows, n_rows, h) != 0 ||
        (k->h_basis == 1 && groth16_gnark_coefficients(k, h) != 0)) {
        free(h);
        return -1;
    }
    msm_outputs_t m;
    groth16_msms(k, w, h, &m);
    free(h);
    if (k->h_basis == 1) {
        fp_t two, half, neg, neg_std;
        fp_from_u64(R, &two, 2);
        fp_inv(R, &half, &two);
        fp_neg(R, &neg, &half);
        fp_from_mont(R, &neg_std, &neg);
        g1j_t t = m.h_g1;
        g1j_mul(&m.h_g1, &t, &neg_std);
    }
    groth16_assemble(k, &m, r, s, p);
    return 0;
}

int groth16_verify(const g1a_t *alpha, const g2a_t *beta, const g2a_t *gamma, const g2a_t *delta,
                   const g1a_t *ic, size_t n_ic, const fp_t *pub, const proof_t *pr) {
    if (pr->a.inf || pr->b.inf || pr->c.inf) return 0;
    if (!g1a_on_curve(&pr->a) || !g1a_on_curve(&pr->c) || !g2a_on_curve(&pr->b)) return 0;
    if (!g2a_in_subgroup(&pr->b)) return 0;
    g1j_t lbar;
    g1j_from_affine(&lbar, &ic[0]);
    for (size_t i = 1; i < n_ic; i++) {
        g1j_t t;
        g1_mul_fr(&t, &ic[i], &pub[i - 1]);
        g1j_add(&lbar, &lbar, &t);
    }
    g1a_t ps[4];
    g2a_t qs[4];
    ps[0] = pr->a;
    fp_neg(&FQ, &ps[0].y, &pr->a.y);
    qs[0] = pr->b;
    ps[1] = *alpha;
    qs[1] = *beta;
    g1j_to_affine(&ps[2], &lbar);
    qs[2] = *gamma;
    ps[3] = pr->c;
    qs[3] = *delta;
    return pairing_product_is_one(ps, qs, 4);
}
