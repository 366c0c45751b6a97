/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Inverses for the timed CPU baseline's batched affine additions: Fermat's
 * little theorem, a^(q-2), over the fast product, and the Fq2 inverse through
 * the norm (a0 - a1 u) / (a0^2 + a1^2).
 */
#include "port_field.h"

static const uint64_t Q_MINUS_2[4] = {PF_Q0 - 2, PF_Q1, PF_Q2, PF_Q3};

void pq_inv(fp_t *r, const fp_t *a) {
    fp_t acc = {{0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL}};
    fp_t base = *a;
    for (int i = 255; i >= 0; i--) {
        pq_mul(&acc, &acc, &acc);
        if ((Q_MINUS_2[i >> 6] >> (i & 63)) & 1) pq_mul(&acc, &acc, &base);
    }
    *r = acc;
}

void pq2_inv(fq2_t *r, const fq2_t *a) {
    fp_t t0, t1, nrm, inv;
    pq_mul(&t0, &a->c0, &a->c0);
    pq_mul(&t1, &a->c1, &a->c1);
    pq_add(&nrm, &t0, &t1);
    pq_inv(&inv, &nrm);
    pq_mul(&r->c0, &a->c0, &inv);
    pq_mul(&t0, &a->c1, &inv);
    pq_neg(&r->c1, &t0);
}
