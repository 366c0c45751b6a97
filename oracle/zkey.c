/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * snarkjs .zkey (Groth16, BN254) reader restating crates/formats/src/lib.rs
 * (ProvingKey::parse :430-505, read_coefficients :905) and
 * crates/formats/src/binfile.rs (:10-26 container, :441-540 decoders):
 *   - iden3 binfile: magic, u32 version, u32 nSections, then
 *     (u32 id, u64 len, payload) entries in any order;
 *   - points: Montgomery little-endian limbs verbatim, (0,0) = infinity,
 *     limbs >= q refused;
 *   - section 4 values: double Montgomery (v R^2), so one Montgomery
 *     multiply by the raw integer 1 yields the Montgomery form of v;
 *   - section 4 sorted by (matrix, constraint) into CSR.
 */
#include "oracle.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { uint32_t id; size_t off, len; } sec_t;

static uint32_t rd32(const uint8_t *b) { uint32_t x; memcpy(&x, b, 4); return x; }
static uint64_t rd64(const uint8_t *b) { uint64_t x; memcpy(&x, b, 8); return x; }

static int fq_raw(fp_t *x, const uint8_t *b) {
    memcpy(x->v, b, 32);
    return fp_lt_modulus(&FQ, x);
}

int unpack_g1(g1a_t *p, const uint8_t *b) {
    if (!fq_raw(&p->x, b) || !fq_raw(&p->y, b + 32)) return 0;
    p->inf = fp_is_zero(&p->x) && fp_is_zero(&p->y);
    return 1;
}

int unpack_g2(g2a_t *p, const uint8_t *b) {
    if (!fq_raw(&p->x.c0, b) || !fq_raw(&p->x.c1, b + 32) || !fq_raw(&p->y.c0, b + 64) ||
        !fq_raw(&p->y.c1, b + 96))
        return 0;
    p->inf = fq2_is_zero(&p->x) && fq2_is_zero(&p->y);
    return 1;
}

void pack_g1(uint8_t *b, const g1a_t *p) {
    if (p->inf) { memset(b, 0, 64); return; }
    memcpy(b, p->x.v, 32);
    memcpy(b + 32, p->y.v, 32);
}

void pack_g2(uint8_t *b, const g2a_t *p) {
    if (p->inf) { memset(b, 0, 128); return; }
    memcpy(b, p->x.c0.v, 32);
    memcpy(b + 32, p->x.c1.v, 32);
    memcpy(b + 64, p->y.c0.v, 32);
    memcpy(b + 96, p->y.c1.v, 32);
}

#define FAIL(...) do { snprintf(err, errlen, __VA_ARGS__); zkey_free(k); free(secs); return -1; } while (0)

static const sec_t *find(const sec_t *s, int ns, uint32_t id) {
    const sec_t *hit = NULL;
    for (int i = 0; i < ns; i++)
        if (s[i].id == id) {
            if (hit) return NULL;   /* duplicate: not unique */
            hit = &s[i];
        }
    return hit;
}

int zkey_parse(zkey_t *k, const uint8_t *d, size_t len, char *err, size_t errlen) {
    memset(k, 0, sizeof *k);
    sec_t *secs = NULL;
    if (len < 12 || memcmp(d, "zkey", 4) != 0) { snprintf(err, errlen, "not a zkey"); return -1; }
    uint32_t nsec = rd32(d + 8);
    if (nsec > 1024) { snprintf(err, errlen, "too many sections"); return -1; }
    secs = calloc(nsec ? nsec : 1, sizeof(sec_t));
    size_t off = 12;
    for (uint32_t i = 0; i < nsec; i++) {
        if (off + 12 > len) FAIL("truncated section header");
        secs[i].id = rd32(d + off);
        uint64_t l = rd64(d + off + 4);
        secs[i].off = off + 12;
        if (l > len - secs[i].off) FAIL("section %u runs past the end", secs[i].id);
        secs[i].len = (size_t)l;
        off = secs[i].off + secs[i].len;
    }
    const sec_t *s1 = find(secs, (int)nsec, 1), *s2 = find(secs, (int)nsec, 2);
    if (!s1 || !s2) FAIL("missing header sections");
    if (s1->len < 4 || rd32(d + s1->off) != 1) FAIL("not groth16");
    const uint8_t *h = d + s2->off;
    size_t hl = s2->len;
    if (hl < 4 + 32 + 4 + 32 + 12 + 64 * 3 + 128 * 3) FAIL("short header");
    if (rd32(h) != 32 || memcmp(h + 4, FQ.p, 32) != 0) FAIL("unsupported curve (q)");
    if (rd32(h + 36) != 32 || memcmp(h + 40, FR.p, 32) != 0) FAIL("unsupported curve (r)");
    k->n_vars = rd32(h + 72);
    k->n_public = rd32(h + 76);
    k->domain_size = rd32(h + 80);
    const uint8_t *pt = h + 84;
    if (!unpack_g1(&k->alpha_g1, pt) || !unpack_g1(&k->beta_g1, pt + 64) ||
        !unpack_g2(&k->beta_g2, pt + 128) || !unpack_g2(&k->gamma_g2, pt + 256) ||
        !unpack_g1(&k->delta_g1, pt + 384) || !unpack_g2(&k->delta_g2, pt + 448))
        FAIL("non-canonical header point");
    uint32_t n = k->domain_size;
    if (n == 0 || (n & (n - 1)) || n > (1u << 27)) FAIL("bad domain size %u", n);
    if (k->n_vars < k->n_public + 1) FAIL("n_vars does not cover 1 + n_public");

    const sec_t *s3 = find(secs, (int)nsec, 3), *s4 = find(secs, (int)nsec, 4);
    const sec_t *s5 = find(secs, (int)nsec, 5), *s6 = find(secs, (int)nsec, 6);
    const sec_t *s7 = find(secs, (int)nsec, 7), *s8 = find(secs, (int)nsec, 8);
    const sec_t *s9 = find(secs, (int)nsec, 9);
    if (!s3 || !s4 || !s5 || !s6 || !s7 || !s8 || !s9) FAIL("missing section");
    size_t nv = k->n_vars, nic = (size_t)k->n_public + 1, nl = nv - nic;
    if (s3->len != nic * 64 || s5->len != nv * 64 || s6->len != nv * 64 || s7->len != nv * 128 ||
        s8->len != nl * 64 || s9->len != (size_t)n * 64)
        FAIL("section length mismatch");
    k->n_ic = nic;
    k->ic = malloc(nic * sizeof(g1a_t));
    k->a_query = malloc(nv * sizeof(g1a_t));
    k->b_g1_query = malloc(nv * sizeof(g1a_t));
    k->b_g2_query = malloc(nv * sizeof(g2a_t));
    k->l_query = malloc((nl ? nl : 1) * sizeof(g1a_t));
    k->h_query = malloc((size_t)n * sizeof(g1a_t));
    k->h_basis = 0;
    k->n_h = n;
    for (size_t i = 0; i < nic; i++) if (!unpack_g1(&k->ic[i], d + s3->off + 64 * i)) FAIL("bad IC point");
    for (size_t i = 0; i < nv; i++) {
        if (!unpack_g1(&k->a_query[i], d + s5->off + 64 * i)) FAIL("bad A point");
        if (!unpack_g1(&k->b_g1_query[i], d + s6->off + 64 * i)) FAIL("bad B1 point");
        if (!unpack_g2(&k->b_g2_query[i], d + s7->off + 128 * i)) FAIL("bad B2 point");
    }
    for (size_t i = 0; i < nl; i++) if (!unpack_g1(&k->l_query[i], d + s8->off + 64 * i)) FAIL("bad C point");
    for (size_t i = 0; i < n; i++) if (!unpack_g1(&k->h_query[i], d + s9->off + 64 * i)) FAIL("bad H point");

    /* section 4: u32 count, then (u32 matrix, u32 constraint, u32 signal, 32 B value) */
    const uint8_t *c4 = d + s4->off;
    if (s4->len < 4) FAIL("short section 4");
    uint32_t ncoef = rd32(c4);
    if ((size_t)ncoef * 44 != s4->len - 4) FAIL("section 4 length mismatch");
    for (int m = 0; m < 2; m++) k->row_ptr[m] = calloc((size_t)n + 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < ncoef; i++) {
        const uint8_t *r = c4 + 4 + 44 * (size_t)i;
        uint32_t m = rd32(r), c = rd32(r + 4), s = rd32(r + 8);
        if (m > 1) FAIL("matrix id %u", m);
        if (c >= n) FAIL("constraint %u outside the domain", c);
        if (s >= k->n_vars) FAIL("signal %u beyond n_vars", s);
        k->row_ptr[m][c + 1]++;
    }
    for (int m = 0; m < 2; m++) {
        for (uint32_t c = 0; c < n; c++) k->row_ptr[m][c + 1] += k->row_ptr[m][c];
        k->nnz[m] = k->row_ptr[m][n];
        k->signal[m] = malloc((k->nnz[m] ? k->nnz[m] : 1) * sizeof(uint32_t));
        k->coef[m] = malloc((k->nnz[m] ? k->nnz[m] : 1) * sizeof(fp_t));
    }
    uint32_t *cur[2];
    for (int m = 0; m < 2; m++) {
        cur[m] = malloc(((size_t)n + 1) * sizeof(uint32_t));
        memcpy(cur[m], k->row_ptr[m], ((size_t)n + 1) * sizeof(uint32_t));
    }
    for (uint32_t i = 0; i < ncoef; i++) {
        const uint8_t *r = c4 + 4 + 44 * (size_t)i;
        uint32_t m = rd32(r), c = rd32(r + 4), s = rd32(r + 8);
        fp_t raw;
        memcpy(raw.v, r + 12, 32);
        if (!fp_lt_modulus(&FR, &raw)) { free(cur[0]); free(cur[1]); FAIL("non-canonical coefficient"); }
        uint32_t at = cur[m][c]++;
        k->signal[m][at] = s;
        fp_from_mont(&FR, &k->coef[m][at], &raw);
    }
    free(cur[0]);
    free(cur[1]);
    free(secs);
    return 0;
}

void zkey_free(zkey_t *k) {
    free(k->ic);
    free(k->a_query);
    free(k->b_g1_query);
    free(k->b_g2_query);
    free(k->l_query);
    free(k->h_query);
    for (int m = 0; m < 2; m++) { free(k->row_ptr[m]); free(k->signal[m]); free(k->coef[m]); }
    memset(k, 0, sizeof *k);
}
