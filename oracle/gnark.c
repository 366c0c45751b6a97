/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * gnark v0.14 Groth16 BN254 files, read into the oracle's key, and the
 * gnark form of stage 9 (the reference's crates/gnark and the
 * HBasis::GnarkBitReversed branch of h_and_msms_from_rows,
 * crates/groth16/src/cpu.rs:384-471, to_gnark_coefficients :265-286):
 *
 *   proving key dump (ProvingKey.WriteDump, crates/gnark/src/pk.rs:1-20):
 *     u64 LE marker 0xdeadbeef; Domain.WriteTo: u64 BE cardinality, five
 *     32-byte BE scalars (1/n, generator, its inverse, the multiplicative
 *     generator and its inverse), one precompute byte; encoder points
 *     G1.Alpha, G1.Beta, G1.Delta, G2.Beta, G2.Delta; u64 BE nbWires,
 *     NbInfinityA, NbInfinityB; the InfinityA and InfinityB flag bytes
 *     (nbWires each); u32 BE commitment count (must be 0); then the dumped
 *     slices G1.A, G1.B, G1.Z, G1.K, G2.B, each a u64 LE count and the points
 *     as Montgomery LE limbs (the packed layout).  G1.A leaves out the wires
 *     flagged in InfinityA, G1.B and G2.B those in InfinityB; G1.Z holds
 *     n - 1 bases for H's coefficients in bit-reversed order; G1.K the
 *     private wires.
 *   verifying key (VerifyingKey.WriteTo / WriteRawTo, crates/gnark/src/vk.rs):
 *     encoder points G1.Alpha, G1.Beta, G2.Beta, G2.Gamma, G1.Delta,
 *     G2.Delta; u32 BE count and the G1.K points (one per public wire,
 *     constant wire first: the IC); u32 BE committed-wire count and u32 BE
 *     commitment count, both 0.
 *   encoder points: big-endian canonical coordinates, X then Y, G2 as A1
 *     then A0; the top two bits of the first byte flag uncompressed (00),
 *     compressed infinity (01), compressed with the smaller (10) or larger
 *     (11) Y, where larger means above (q - 1) / 2, for Fq2 by A1 unless it
 *     is zero, then by A0.
 */
#include "oracle.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define Q (&FQ)
#define R (&FR)

typedef struct {
    const uint8_t *d;
    size_t len, pos;
    char *err;
    size_t errlen;
} rd_t;

static int take(rd_t *r, size_t n, const uint8_t **out) {
    if (n > r->len - r->pos) {
        snprintf(r->err, r->errlen, "truncated at offset %zu (wanted %zu bytes)", r->pos, n);
        return -1;
    }
    *out = r->d + r->pos;
    r->pos += n;
    return 0;
}

static int be64(rd_t *r, uint64_t *v) {
    const uint8_t *b;
    if (take(r, 8, &b)) return -1;
    *v = 0;
    for (int i = 0; i < 8; i++) *v = (*v << 8) | b[i];
    return 0;
}

static int be32(rd_t *r, uint32_t *v) {
    const uint8_t *b;
    if (take(r, 4, &b)) return -1;
    *v = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
    return 0;
}

static int le64(rd_t *r, uint64_t *v) {
    const uint8_t *b;
    if (take(r, 8, &b)) return -1;
    *v = 0;
    for (int i = 7; i >= 0; i--) *v = (*v << 8) | b[i];
    return 0;
}

/* 32 big-endian bytes -> Montgomery element of f, refused at or above the modulus */
static int be_elem(const field_t *f, const uint8_t *b, fp_t *out) {
    fp_t raw;
    for (int l = 0; l < 4; l++) {
        uint64_t v = 0;
        for (int i = 0; i < 8; i++) v = (v << 8) | b[(3 - l) * 8 + i];
        raw.v[l] = v;
    }
    if (!fp_lt_modulus(f, &raw)) return -1;
    fp_to_mont(f, out, &raw);
    return 0;
}

static int fq_larger(const fp_t *y_mont) {
    /* above (q - 1) / 2 as an integer */
    fp_t y, half;
    fp_from_mont(Q, &y, y_mont);
    /* half = (q - 1) / 2: q is odd, so a right shift of q */
    for (int l = 0; l < 4; l++) {
        half.v[l] = FQ.p[l] >> 1;
        if (l < 3) half.v[l] |= FQ.p[l + 1] << 63;
    }
    for (int l = 3; l >= 0; l--)
        if (y.v[l] != half.v[l]) return y.v[l] > half.v[l];
    return 0;
}

static int encoder_g1(rd_t *r, g1a_t *p) {
    const uint8_t *b;
    if (take(r, 32, &b)) return -1;
    const int flag = b[0] >> 6;
    uint8_t x[32];
    memcpy(x, b, 32);
    x[0] &= 0x3f;
    memset(p, 0, sizeof *p);
    if (flag == 1) { p->inf = 1; return 0; }
    if (be_elem(Q, x, &p->x)) { snprintf(r->err, r->errlen, "G1 x not canonical"); return -1; }
    if (flag == 0) {
        const uint8_t *yb;
        if (take(r, 32, &yb)) return -1;
        static const uint8_t zero[32];
        if (!memcmp(x, zero, 32) && !memcmp(yb, zero, 32)) { p->inf = 1; return 0; }
        if (be_elem(Q, yb, &p->y)) { snprintf(r->err, r->errlen, "G1 y not canonical"); return -1; }
    } else {
        fp_t y2, t, three;
        fp_sqr(Q, &t, &p->x);
        fp_mul(Q, &y2, &t, &p->x);
        fp_from_u64(Q, &three, 3);
        fp_add(Q, &y2, &y2, &three);
        if (!fp_sqrt(Q, &p->y, &y2)) { snprintf(r->err, r->errlen, "compressed G1 x off the curve"); return -1; }
        if (fq_larger(&p->y) != (flag == 3)) fp_neg(Q, &p->y, &p->y);
    }
    if (!g1a_on_curve(p)) { snprintf(r->err, r->errlen, "G1 point off the curve"); return -1; }
    return 0;
}

static int encoder_g2(rd_t *r, g2a_t *p) {
    const uint8_t *b;
    if (take(r, 64, &b)) return -1;
    const int flag = b[0] >> 6;
    uint8_t x1[32];
    memcpy(x1, b, 32);
    x1[0] &= 0x3f;
    memset(p, 0, sizeof *p);
    if (flag == 1) { p->inf = 1; return 0; }
    if (be_elem(Q, x1, &p->x.c1) || be_elem(Q, b + 32, &p->x.c0)) {
        snprintf(r->err, r->errlen, "G2 x not canonical");
        return -1;
    }
    if (flag == 0) {
        const uint8_t *yb;
        if (take(r, 64, &yb)) return -1;
        static const uint8_t zero[64];
        if (!memcmp(b, zero, 64) && !memcmp(yb, zero, 64)) { p->inf = 1; return 0; }
        if (be_elem(Q, yb, &p->y.c1) || be_elem(Q, yb + 32, &p->y.c0)) {
            snprintf(r->err, r->errlen, "G2 y not canonical");
            return -1;
        }
    } else {
        fq2_t y2, t, b2, xi, xi_inv, three = {{{0}}, {{0}}};
        fp_from_u64(Q, &three.c0, 3);   /* b' = 3 / (9 + u) */
        fp_from_u64(Q, &xi.c0, 9);
        fp_from_u64(Q, &xi.c1, 1);
        fq2_inv(&xi_inv, &xi);
        fq2_mul(&b2, &three, &xi_inv);
        fq2_sqr(&t, &p->x);
        fq2_mul(&y2, &t, &p->x);
        fq2_add(&y2, &y2, &b2);
        if (!fq2_sqrt(&p->y, &y2)) { snprintf(r->err, r->errlen, "compressed G2 x off the curve"); return -1; }
        const int larger = fp_is_zero(&p->y.c1) ? fq_larger(&p->y.c0) : fq_larger(&p->y.c1);
        if (larger != (flag == 3)) fq2_neg(&p->y, &p->y);
    }
    if (!g2a_on_curve(p)) { snprintf(r->err, r->errlen, "G2 point off the curve"); return -1; }
    return 0;
}

/* a dumped slice: u64 LE count, count records of stride bytes */
static int dumped(rd_t *r, size_t stride, const uint8_t **data, size_t *count) {
    uint64_t n;
    if (le64(r, &n)) return -1;
    if (n > (r->len - r->pos) / stride) {
        snprintf(r->err, r->errlen, "dumped slice of %llu records does not fit", (unsigned long long)n);
        return -1;
    }
    *count = (size_t)n;
    return take(r, (size_t)n * stride, data);
}

static int same_g1(const g1a_t *a, const g1a_t *b) { return g1a_eq(a, b); }
static int same_g2(const g2a_t *a, const g2a_t *b) {
    if (a->inf || b->inf) return a->inf == b->inf;
    return fq2_eq(&a->x, &b->x) && fq2_eq(&a->y, &b->y);
}

#define FAIL(...) do { snprintf(err, errlen, __VA_ARGS__); zkey_free(k); return -1; } while (0)

int gnark_parse(zkey_t *k, const uint8_t *pk, size_t pk_len, const uint8_t *vk, size_t vk_len, char *err,
                size_t errlen) {
    bn254_init();
    memset(k, 0, sizeof *k);
    rd_t r = {pk, pk_len, 0, err, errlen};
    const uint8_t *b;
    static const uint8_t marker[8] = {0xef, 0xbe, 0xad, 0xde, 0, 0, 0, 0};
    if (take(&r, 8, &b) || memcmp(b, marker, 8)) FAIL("not a gnark dump (marker)");
    uint64_t card;
    if (be64(&r, &card)) return zkey_free(k), -1;
    if (card < 2 || (card & (card - 1)) || card > (1ull << 27)) FAIL("domain cardinality %llu", (unsigned long long)card);
    int log_n = 0;
    while ((1ull << log_n) < card) log_n++;
    fp_t dom[5];
    for (int i = 0; i < 5; i++) {
        if (take(&r, 32, &b) || be_elem(R, b, &dom[i])) FAIL("domain scalar %d", i);
    }
    fp_t omega, ninv, n_fr;
    domain_root(log_n, &omega);
    fp_from_u64(R, &n_fr, card);
    fp_inv(R, &ninv, &n_fr);
    if (!fp_eq(&dom[0], &ninv) || !fp_eq(&dom[1], &omega)) FAIL("domain is not the one for 2^%d", log_n);
    if (take(&r, 1, &b) || b[0] > 1) FAIL("precompute byte");
    g1a_t alpha, beta1, delta1;
    g2a_t beta2, delta2;
    if (encoder_g1(&r, &alpha) || encoder_g1(&r, &beta1) || encoder_g1(&r, &delta1) || encoder_g2(&r, &beta2) ||
        encoder_g2(&r, &delta2))
        return zkey_free(k), -1;
    uint64_t nw, ninf_a, ninf_b;
    if (be64(&r, &nw) || be64(&r, &ninf_a) || be64(&r, &ninf_b)) return zkey_free(k), -1;
    if (nw > r.len || nw < 1) FAIL("%llu wires", (unsigned long long)nw);
    const uint8_t *flag_a, *flag_b;
    if (take(&r, nw, &flag_a) || take(&r, nw, &flag_b)) return zkey_free(k), -1;
    uint64_t ca = 0, cb = 0;
    for (uint64_t i = 0; i < nw; i++) {
        if (flag_a[i] > 1 || flag_b[i] > 1) FAIL("infinity flag %llu not a bool", (unsigned long long)i);
        ca += flag_a[i];
        cb += flag_b[i];
    }
    if (ca != ninf_a || cb != ninf_b) FAIL("infinity flag counts");
    uint32_t ncommit;
    if (be32(&r, &ncommit)) return zkey_free(k), -1;
    if (ncommit) FAIL("%u commitment keys", ncommit);
    const uint8_t *sa, *sb, *sz, *sk, *sb2;
    size_t na, nb, nz, nk, nb2;
    if (dumped(&r, 64, &sa, &na) || dumped(&r, 64, &sb, &nb) || dumped(&r, 64, &sz, &nz) ||
        dumped(&r, 64, &sk, &nk) || dumped(&r, 128, &sb2, &nb2))
        return zkey_free(k), -1;
    if (r.pos != r.len) FAIL("%zu trailing bytes", r.len - r.pos);
    if (na != nw - ca || nb != nw - cb || nb2 != nw - cb || nz != card - 1 || nk >= nw) FAIL("slice lengths");

    /* verifying key */
    rd_t v = {vk, vk_len, 0, err, errlen};
    g1a_t valpha, vbeta1, vdelta1;
    g2a_t vbeta2, vgamma2, vdelta2;
    if (encoder_g1(&v, &valpha) || encoder_g1(&v, &vbeta1) || encoder_g2(&v, &vbeta2) || encoder_g2(&v, &vgamma2) ||
        encoder_g1(&v, &vdelta1) || encoder_g2(&v, &vdelta2))
        return zkey_free(k), -1;
    if (!same_g1(&valpha, &alpha) || !same_g1(&vbeta1, &beta1) || !same_g1(&vdelta1, &delta1) ||
        !same_g2(&vbeta2, &beta2) || !same_g2(&vdelta2, &delta2))
        FAIL("verifying key and proving key differ");
    uint32_t nic;
    if (be32(&v, &nic)) return zkey_free(k), -1;
    if (nic != nw - nk || nic < 1) FAIL("verifying key has %u K points for %llu public wires", nic,
                                        (unsigned long long)(nw - nk));
    k->ic = calloc(nic, sizeof(g1a_t));
    k->n_ic = nic;
    for (uint32_t i = 0; i < nic; i++)
        if (encoder_g1(&v, &k->ic[i])) return zkey_free(k), -1;
    uint32_t c1, c2;
    if (be32(&v, &c1) || be32(&v, &c2)) return zkey_free(k), -1;
    if (c1 || c2 || v.pos != v.len) FAIL("verifying key commitments or trailing bytes");

    k->n_vars = (uint32_t)nw;
    k->n_public = nic - 1;
    k->domain_size = (uint32_t)card;
    k->alpha_g1 = alpha;
    k->beta_g1 = beta1;
    k->delta_g1 = delta1;
    k->beta_g2 = beta2;
    k->gamma_g2 = vgamma2;
    k->delta_g2 = delta2;
    k->h_basis = 1;
    k->n_h = card - 1;
    k->a_query = calloc(nw, sizeof(g1a_t));
    k->b_g1_query = calloc(nw, sizeof(g1a_t));
    k->b_g2_query = calloc(nw, sizeof(g2a_t));
    k->l_query = calloc(nk ? nk : 1, sizeof(g1a_t));
    k->h_query = calloc(nz, sizeof(g1a_t));
    size_t ia = 0, ib = 0;
    for (uint64_t i = 0; i < nw; i++) {
        if (flag_a[i]) k->a_query[i].inf = 1;
        else if (!unpack_g1(&k->a_query[i], sa + 64 * ia++)) FAIL("G1.A point");
        if (flag_b[i]) {
            k->b_g1_query[i].inf = 1;
            k->b_g2_query[i].inf = 1;
        } else {
            if (!unpack_g1(&k->b_g1_query[i], sb + 64 * ib) || !unpack_g2(&k->b_g2_query[i], sb2 + 128 * ib))
                FAIL("G1.B / G2.B point");
            ib++;
        }
    }
    for (size_t i = 0; i < nk; i++)
        if (!unpack_g1(&k->l_query[i], sk + 64 * i)) FAIL("G1.K point");
    for (size_t i = 0; i < nz; i++)
        if (!unpack_g1(&k->h_query[i], sz + 64 * i)) FAIL("G1.Z point");
    return 0;
}

/* H on the odd coset -> H's coefficients in bit-reversed order, the form
 * gnark's Z bases take (to_gnark_coefficients, crates/groth16/src/cpu.rs:265-286):
 * the inverse coset transform gives the coefficients c_j of the polynomial
 * whose values on the coset are h, which is (-2) H since t = x^n - 1 is -2
 * there; the -1/2 is applied to the MSM result.  Refused unless coefficient
 * n - 1 is zero, as it is for any witness when the arithmetic is right. */
int groth16_gnark_coefficients(const zkey_t *k, fp_t *h) {
    domain_t d;
    int log_n = 0;
    while ((1u << log_n) < k->domain_size) log_n++;
    if (domain_init(&d, log_n)) return -1;
    ntt_inverse(&d, h);
    fp_t shift_inv;
    fp_inv(R, &shift_inv, &d.shift);
    distribute_powers(h, d.n, &shift_inv);
    bitrev_permute(h, d.n);
    const int ok = fp_is_zero(&h[d.n - 1]);
    domain_free(&d);
    return ok ? 0 : -1;
}
