/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * The timed CPU baseline's prover: stages 0-9 of CpuCircuit::h_and_msms
 * (crates/groth16/src/cpu.rs:316-382, 477-632) over the port's field, NTT and
 * MSM, scheduled as the reference schedules them:
 *   - stage 0: the A and B gathers concurrently, each parallel over rows,
 *     zero witness values skipped and ones added without a product
 *     (cpu.rs:140-174, 321-337), then C = A * B;
 *   - stages 1-3: the three intt_coset_ntt concurrently (cpu.rs:191-227);
 *   - stage 4: H = A * B - C in place (cpu.rs:236-246);
 *   - stages 5-9: the five MSMs concurrently (cpu.rs:585-621);
 *   - stage 11: the oracle's blinding and assembly (prove.rs:335-430).
 * The proof equals the oracle's (groth16.c) for the same witness, r and s.
 */
#include "port.h"
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ROW_CHUNK 8192

static int fr_is_one(const fp_t *a) { return pf_eq(a, &FR.one); }

static void gather_tasks(const zkey_t *k, int m, const fp_t *w, fp_t *out) {
    const size_t n = k->domain_size;
    const uint32_t *rp = k->row_ptr[m], *sg = k->signal[m];
    const fp_t *cf = k->coef[m];
#pragma omp taskloop num_tasks(port_tasks())
    for (size_t t = 0; t < (n + ROW_CHUNK - 1) / ROW_CHUNK; t++) {
        size_t lo = t * ROW_CHUNK, hi = lo + ROW_CHUNK < n ? lo + ROW_CHUNK : n;
        for (size_t row = lo; row < hi; row++) {
            fp_t acc = {{0, 0, 0, 0}};
            for (uint32_t e = rp[row]; e < rp[row + 1]; e++) {
                const fp_t *x = &w[sg[e]];
                if (pf_is_zero(x)) continue;
                if (fr_is_one(x)) {
                    pr_add(&acc, &acc, &cf[e]);
                } else {
                    fp_t prod;
                    pr_mul(&prod, &cf[e], x);
                    pr_add(&acc, &acc, &prod);
                }
            }
            out[row] = acc;
        }
    }
}

static void from_mont_tasks(fp_t *out, const fp_t *in, size_t n) {
    static const fp_t one_std = {{1, 0, 0, 0}};
#pragma omp taskloop num_tasks(port_tasks())
    for (size_t t = 0; t < (n + ROW_CHUNK - 1) / ROW_CHUNK; t++) {
        size_t lo = t * ROW_CHUNK, hi = lo + ROW_CHUNK < n ? lo + ROW_CHUNK : n;
        for (size_t i = lo; i < hi; i++) pr_mul(&out[i], &in[i], &one_std);
    }
}

int port_prove(const zkey_t *k, const port_ntt *t, const fp_t *w, const fp_t *r, const fp_t *s, proof_t *p) {
    const size_t n = k->domain_size, nv = k->n_vars, off = (size_t)k->n_public + 1;
    fp_t *a = malloc(n * sizeof(fp_t)), *b = malloc(n * sizeof(fp_t)), *c = malloc(n * sizeof(fp_t));
    fp_t *ws = malloc(nv * sizeof(fp_t));
    if (!a || !b || !c || !ws) {
        free(a); free(b); free(c); free(ws);
        return -1;
    }
    msm_outputs_t m;
    int threads = 1;
#ifdef _OPENMP
    threads = omp_get_max_threads();
#endif
#pragma omp parallel
#pragma omp single
    {
        /* stage 0 */
#pragma omp taskgroup
        {
#pragma omp task
            gather_tasks(k, 0, w, a);
#pragma omp task
            gather_tasks(k, 1, w, b);
        }
#pragma omp taskloop num_tasks(port_tasks())
        for (size_t q = 0; q < (n + ROW_CHUNK - 1) / ROW_CHUNK; q++) {
            size_t lo = q * ROW_CHUNK, hi = lo + ROW_CHUNK < n ? lo + ROW_CHUNK : n;
            for (size_t i = lo; i < hi; i++) pr_mul(&c[i], &a[i], &b[i]);
        }
        /* stages 1-3, the three vectors concurrently */
#pragma omp taskgroup
        {
#pragma omp task
            port_intt_coset_ntt_tasks(t, a);
#pragma omp task
            port_intt_coset_ntt_tasks(t, b);
#pragma omp task
            port_intt_coset_ntt_tasks(t, c);
        }
        /* stage 4: H = A B - C into a */
#pragma omp taskloop num_tasks(port_tasks())
        for (size_t q = 0; q < (n + ROW_CHUNK - 1) / ROW_CHUNK; q++) {
            size_t lo = q * ROW_CHUNK, hi = lo + ROW_CHUNK < n ? lo + ROW_CHUNK : n;
            for (size_t i = lo; i < hi; i++) {
                fp_t x;
                pr_mul(&x, &a[i], &b[i]);
                pr_sub(&a[i], &x, &c[i]);
            }
        }
        /* stages 5-9: scalars to standard form, then the five MSMs concurrently */
#pragma omp taskgroup
        {
#pragma omp task
            from_mont_tasks(ws, w, nv);
#pragma omp task
            from_mont_tasks(b, a, n);
        }
#pragma omp taskgroup
        {
#pragma omp task
            port_msm_g1_tasks(&m.a_g1, k->a_query, ws, nv, threads);
#pragma omp task
            port_msm_g2_tasks(&m.b_g2, k->b_g2_query, ws, nv, threads);
#pragma omp task
            port_msm_g1_tasks(&m.b_g1, k->b_g1_query, ws, nv, threads);
#pragma omp task
            port_msm_g1_tasks(&m.l_g1, k->l_query, ws + off, nv - off, threads);
#pragma omp task
            port_msm_g1_tasks(&m.h_g1, k->h_query, b, n, threads);
        }
    }
    groth16_assemble(k, &m, r, s, p);
    free(a);
    free(b);
    free(c);
    free(ws);
    return 0;
}
