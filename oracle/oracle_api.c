/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Flat byte-buffer entry points for the Python tests (ctypes).  Field
 * elements are 32-byte little-endian; Fr/Fq values are Montgomery form
 * unless a name says _std.  Points use the packed layout of snarkrs'
 * gpu-layout crate (crates/gpu-layout/src/lib.rs:120-200, 351): G1 = x||y,
 * G2 = x.c0||x.c1||y.c0||y.c1, infinity = all-zero bytes.
 * A proof is A(64) || B(128) || C(64).
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define R (&FR)

static void ld(fp_t *x, const uint8_t *b) { memcpy(x->v, b, 32); }
static void st(uint8_t *b, const fp_t *x) { memcpy(b, x->v, 32); }

void oracle_init(void) { bn254_init(); }

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---- field ---- */
static const field_t *fld(int which) { return which ? &FQ : &FR; }
void oracle_fp_mul(int which, const uint8_t *a, const uint8_t *b, uint8_t *out) {
    fp_t x, y, z; ld(&x, a); ld(&y, b); fp_mul(fld(which), &z, &x, &y); st(out, &z);
}
void oracle_fp_add(int which, const uint8_t *a, const uint8_t *b, uint8_t *out) {
    fp_t x, y, z; ld(&x, a); ld(&y, b); fp_add(fld(which), &z, &x, &y); st(out, &z);
}
void oracle_fp_sub(int which, const uint8_t *a, const uint8_t *b, uint8_t *out) {
    fp_t x, y, z; ld(&x, a); ld(&y, b); fp_sub(fld(which), &z, &x, &y); st(out, &z);
}
void oracle_fp_inv(int which, const uint8_t *a, uint8_t *out) {
    fp_t x, z; ld(&x, a); fp_inv(fld(which), &z, &x); st(out, &z);
}
void oracle_fp_to_mont(int which, const uint8_t *a, uint8_t *out) {
    fp_t x, z; ld(&x, a); fp_to_mont(fld(which), &z, &x); st(out, &z);
}
void oracle_fp_from_mont(int which, const uint8_t *a, uint8_t *out) {
    fp_t x, z; ld(&x, a); fp_from_mont(fld(which), &z, &x); st(out, &z);
}
void oracle_field_consts(int which, uint8_t *p, uint64_t *n0, uint8_t *one, uint8_t *r2) {
    const field_t *f = fld(which);
    memcpy(p, f->p, 32);
    *n0 = f->n0;
    st(one, &f->one);
    st(r2, &f->r2);
}
void oracle_fq2_mul(const uint8_t *a, const uint8_t *b, uint8_t *out) {
    fq2_t x, y, z;
    ld(&x.c0, a); ld(&x.c1, a + 32); ld(&y.c0, b); ld(&y.c1, b + 32);
    fq2_mul(&z, &x, &y);
    st(out, &z.c0); st(out + 32, &z.c1);
}

int oracle_hard_exponent(uint32_t *out40);

/* ---- domain and NTT ---- */
int oracle_domain_root(int log_n, uint8_t *out) {
    fp_t w;
    if (domain_root(log_n, &w) != 0) return -1;
    st(out, &w);
    return 0;
}

/* mode 0 forward, 1 inverse, 2 intt_coset_ntt, 3 coset forward
 * (a[i] *= shift^i then forward; shift = the proving coset shift when
 * shift_mont is NULL), 4 coset inverse (inverse then a[i] *= shift^-i) */
int oracle_ntt(int log_n, int mode, uint8_t *data, const uint8_t *shift_mont) {
    domain_t d;
    if (domain_init(&d, log_n) != 0) return -1;
    fp_t *a = (fp_t *)data;   /* fp_t is exactly 32 packed bytes */
    fp_t shift = d.shift;
    if (shift_mont) ld(&shift, shift_mont);
    switch (mode) {
    case 0: ntt_forward(&d, a); break;
    case 1: ntt_inverse(&d, a); break;
    case 2: intt_coset_ntt(&d, a); break;
    case 3: distribute_powers(a, d.n, &shift); ntt_forward(&d, a); break;
    case 4: {
        fp_t si;
        fp_inv(R, &si, &shift);
        ntt_inverse(&d, a);
        distribute_powers(a, d.n, &si);
        break;
    }
    default: domain_free(&d); return -1;
    }
    domain_free(&d);
    return 0;
}

/* ---- curve ---- */
void oracle_g1_generator(uint8_t *out) { pack_g1(out, &G1_GEN); }
void oracle_g2_generator(uint8_t *out) { pack_g2(out, &G2_GEN); }

int oracle_g1_mul(const uint8_t *p, const uint8_t *k_std, uint8_t *out) {
    g1a_t a; fp_t k; g1j_t j, r;
    if (!unpack_g1(&a, p)) return -1;
    ld(&k, k_std);
    g1j_from_affine(&j, &a);
    g1j_mul(&r, &j, &k);
    g1j_to_affine(&a, &r);
    pack_g1(out, &a);
    return 0;
}
int oracle_g2_mul(const uint8_t *p, const uint8_t *k_std, uint8_t *out) {
    g2a_t a; fp_t k; g2j_t j, r;
    if (!unpack_g2(&a, p)) return -1;
    ld(&k, k_std);
    g2j_from_affine(&j, &a);
    g2j_mul(&r, &j, &k);
    g2j_to_affine(&a, &r);
    pack_g2(out, &a);
    return 0;
}
int oracle_g1_add(const uint8_t *p, const uint8_t *q, uint8_t *out) {
    g1a_t a, b; g1j_t j, r;
    if (!unpack_g1(&a, p) || !unpack_g1(&b, q)) return -1;
    g1j_from_affine(&j, &a);
    g1j_add_affine(&r, &j, &b);
    g1j_to_affine(&a, &r);
    pack_g1(out, &a);
    return 0;
}
int oracle_g2_add(const uint8_t *p, const uint8_t *q, uint8_t *out) {
    g2a_t a, b; g2j_t j, r;
    if (!unpack_g2(&a, p) || !unpack_g2(&b, q)) return -1;
    g2j_from_affine(&j, &a);
    g2j_add_affine(&r, &j, &b);
    g2j_to_affine(&a, &r);
    pack_g2(out, &a);
    return 0;
}
int oracle_g1_on_curve(const uint8_t *p) { g1a_t a; return unpack_g1(&a, p) && g1a_on_curve(&a); }
int oracle_g2_on_curve(const uint8_t *p) { g2a_t a; return unpack_g2(&a, p) && g2a_on_curve(&a); }
int oracle_g2_in_subgroup(const uint8_t *p) { g2a_t a; return unpack_g2(&a, p) && g2a_in_subgroup(&a); }

/* ---- MSM (scalars in standard form) ---- */
int oracle_msm_g1(const uint8_t *bases, const uint8_t *scalars_std, size_t n, uint8_t *out) {
    g1a_t *b = malloc((n ? n : 1) * sizeof(g1a_t));
    for (size_t i = 0; i < n; i++) if (!unpack_g1(&b[i], bases + 64 * i)) { free(b); return -1; }
    g1j_t r;
    msm_g1(&r, b, (const fp_t *)scalars_std, n);
    g1a_t a;
    g1j_to_affine(&a, &r);
    pack_g1(out, &a);
    free(b);
    return 0;
}
int oracle_msm_g2(const uint8_t *bases, const uint8_t *scalars_std, size_t n, uint8_t *out) {
    g2a_t *b = malloc((n ? n : 1) * sizeof(g2a_t));
    for (size_t i = 0; i < n; i++) if (!unpack_g2(&b[i], bases + 128 * i)) { free(b); return -1; }
    g2j_t r;
    msm_g2(&r, b, (const fp_t *)scalars_std, n);
    g2a_t a;
    g2j_to_affine(&a, &r);
    pack_g2(out, &a);
    free(b);
    return 0;
}

/* ---- zkey and prover ---- */
void *oracle_zkey_load(const uint8_t *bytes, size_t len, char *err, size_t errlen) {
    zkey_t *k = malloc(sizeof *k);
    if (zkey_parse(k, bytes, len, err, errlen) != 0) { free(k); return NULL; }
    return k;
}
void oracle_zkey_free(void *k) { if (k) { zkey_free(k); free(k); } }
void oracle_zkey_info(const void *kv, uint32_t *out3) {
    const zkey_t *k = kv;
    out3[0] = k->n_vars; out3[1] = k->n_public; out3[2] = k->domain_size;
}

int oracle_gather(const void *kv, const uint8_t *w_mont, size_t n, uint8_t *a_out, uint8_t *b_out) {
    const zkey_t *k = kv;
    if (n != k->n_vars) return -1;
    groth16_gather(k, (const fp_t *)w_mont, (fp_t *)a_out, (fp_t *)b_out);
    return 0;
}

int oracle_compute_h_from_rows(const void *kv, const uint8_t *a_rows, const uint8_t *b_rows, size_t rows,
                               uint8_t *h_out) {
    return groth16_compute_h_from_rows(kv, (const fp_t *)a_rows, (const fp_t *)b_rows, rows, (fp_t *)h_out);
}

int oracle_compute_h(const void *kv, const uint8_t *w_mont, size_t n, uint8_t *h_out) {
    const zkey_t *k = kv;
    if (n != k->n_vars) return -1;
    return groth16_compute_h(k, (const fp_t *)w_mont, (fp_t *)h_out);
}

/* out: A(64) || B2(128) || B1(64) || L(64) || H(64), affine packed */
int oracle_msms(const void *kv, const uint8_t *w_mont, size_t n, const uint8_t *h_mont, uint8_t *out) {
    const zkey_t *k = kv;
    if (n != k->n_vars) return -1;
    msm_outputs_t m;
    groth16_msms(k, (const fp_t *)w_mont, (const fp_t *)h_mont, &m);
    g1a_t a; g2a_t b;
    g1j_to_affine(&a, &m.a_g1); pack_g1(out, &a);
    g2j_to_affine(&b, &m.b_g2); pack_g2(out + 64, &b);
    g1j_to_affine(&a, &m.b_g1); pack_g1(out + 192, &a);
    g1j_to_affine(&a, &m.l_g1); pack_g1(out + 256, &a);
    g1j_to_affine(&a, &m.h_g1); pack_g1(out + 320, &a);
    return 0;
}

static void pack_proof(uint8_t *out, const proof_t *p) {
    pack_g1(out, &p->a);
    pack_g2(out + 64, &p->b);
    pack_g1(out + 192, &p->c);
}

void *oracle_gnark_load(const uint8_t *pk, size_t pk_len, const uint8_t *vk, size_t vk_len, char *err,
                        size_t errlen) {
    zkey_t *k = calloc(1, sizeof *k);
    if (gnark_parse(k, pk, pk_len, vk, vk_len, err, errlen) != 0) {
        free(k);
        return NULL;
    }
    return k;
}

int oracle_zkey_h_basis(const void *kv) { return ((const zkey_t *)kv)->h_basis; }

/* one query packed (0 A, 1 B1, 2 B2, 3 L, 4 H), returns its point count; out NULL sizes */
size_t oracle_zkey_query(const void *kv, int which, uint8_t *out) {
    const zkey_t *k = kv;
    const size_t nv = k->n_vars, nl = nv - k->n_public - 1, nh = k->n_h ? k->n_h : k->domain_size;
    const size_t n = which == 3 ? nl : which == 4 ? nh : nv;
    if (out)
        for (size_t i = 0; i < n; i++) {
            if (which == 2) pack_g2(out + 128 * i, &k->b_g2_query[i]);
            else pack_g1(out + 64 * i, which == 0 ? &k->a_query[i] : which == 1 ? &k->b_g1_query[i]
                                       : which == 3 ? &k->l_query[i] : &k->h_query[i]);
        }
    return n;
}

/* alpha_g1 | beta_g2 | gamma_g2 | delta_g2 | ic..., packed */
size_t oracle_zkey_vk(const void *kv, uint8_t *out) {
    const zkey_t *k = kv;
    if (out) {
        pack_g1(out, &k->alpha_g1);
        pack_g2(out + 64, &k->beta_g2);
        pack_g2(out + 192, &k->gamma_g2);
        pack_g2(out + 320, &k->delta_g2);
        for (size_t i = 0; i < k->n_ic; i++) pack_g1(out + 448 + 64 * i, &k->ic[i]);
    }
    return 448 + 64 * k->n_ic;
}

int oracle_prove_rows(const void *kv, const uint8_t *w_mont, size_t n, const uint8_t *a_rows, const uint8_t *b_rows,
                      size_t rows, const uint8_t *r_mont, const uint8_t *s_mont, uint8_t *proof_out) {
    const zkey_t *k = kv;
    if (n != k->n_vars) return -1;
    fp_t r, s;
    ld(&r, r_mont); ld(&s, s_mont);
    proof_t p;
    if (groth16_prove_rows(k, (const fp_t *)w_mont, (const fp_t *)a_rows, (const fp_t *)b_rows, rows, &r, &s, &p) != 0)
        return -1;
    pack_proof(proof_out, &p);
    return 0;
}

int oracle_prove(const void *kv, const uint8_t *w_mont, size_t n, const uint8_t *r_mont,
                 const uint8_t *s_mont, uint8_t *proof_out) {
    const zkey_t *k = kv;
    if (n != k->n_vars) return -1;
    fp_t r, s;
    ld(&r, r_mont); ld(&s, s_mont);
    proof_t p;
    if (groth16_prove(k, (const fp_t *)w_mont, &r, &s, &p) != 0) return -1;
    pack_proof(proof_out, &p);
    return 0;
}

int oracle_verify_zkey(const void *kv, const uint8_t *pub_mont, size_t n_pub, const uint8_t *proof) {
    const zkey_t *k = kv;
    if (n_pub != k->n_public) return -1;
    proof_t p;
    if (!unpack_g1(&p.a, proof) || !unpack_g2(&p.b, proof + 64) || !unpack_g1(&p.c, proof + 192)) return 0;
    return groth16_verify(&k->alpha_g1, &k->beta_g2, &k->gamma_g2, &k->delta_g2, k->ic, k->n_ic,
                          (const fp_t *)pub_mont, &p);
}

/* vk given as packed points: alpha(64) beta(128) gamma(128) delta(128) then ic[n_ic](64 each) */
int oracle_verify_vk(const uint8_t *vk, size_t n_ic, const uint8_t *pub_mont, const uint8_t *proof) {
    g1a_t alpha; g2a_t beta, gamma, delta;
    if (!unpack_g1(&alpha, vk) || !unpack_g2(&beta, vk + 64) || !unpack_g2(&gamma, vk + 192) ||
        !unpack_g2(&delta, vk + 320))
        return -1;
    g1a_t *ic = malloc(n_ic * sizeof(g1a_t));
    for (size_t i = 0; i < n_ic; i++)
        if (!unpack_g1(&ic[i], vk + 448 + 64 * i)) { free(ic); return -1; }
    proof_t p;
    int ok = unpack_g1(&p.a, proof) && unpack_g2(&p.b, proof + 64) && unpack_g1(&p.c, proof + 192);
    if (ok) ok = groth16_verify(&alpha, &beta, &gamma, &delta, ic, n_ic, (const fp_t *)pub_mont, &p);
    free(ic);
    return ok;
}

/* e(p1,q1) e(p2,q2) ... == 1 */
int oracle_pairing_check(const uint8_t *g1s, const uint8_t *g2s, int n) {
    g1a_t *p = malloc(n * sizeof(g1a_t));
    g2a_t *q = malloc(n * sizeof(g2a_t));
    for (int i = 0; i < n; i++)
        if (!unpack_g1(&p[i], g1s + 64 * i) || !unpack_g2(&q[i], g2s + 128 * i)) { free(p); free(q); return -1; }
    int r = pairing_product_is_one(p, q, n);
    free(p);
    free(q);
    return r;
}

/* ---- the timed CPU baseline (port_*.c): same results, the reference's fast algorithms ---- */
#include "port.h"

int oracle_port_msm_g1(const uint8_t *bases, const uint8_t *scalars_std, size_t n, uint8_t *out) {
    g1a_t *b = malloc((n ? n : 1) * sizeof(g1a_t));
    for (size_t i = 0; i < n; i++) if (!unpack_g1(&b[i], bases + 64 * i)) { free(b); return -1; }
    g1j_t r;
    port_msm_g1(&r, b, (const fp_t *)scalars_std, n);
    g1a_t a;
    g1j_to_affine(&a, &r);
    pack_g1(out, &a);
    free(b);
    return 0;
}

int oracle_port_msm_g2(const uint8_t *bases, const uint8_t *scalars_std, size_t n, uint8_t *out) {
    g2a_t *b = malloc((n ? n : 1) * sizeof(g2a_t));
    for (size_t i = 0; i < n; i++) if (!unpack_g2(&b[i], bases + 128 * i)) { free(b); return -1; }
    g2j_t r;
    port_msm_g2(&r, b, (const fp_t *)scalars_std, n);
    g2a_t a;
    g2j_to_affine(&a, &r);
    pack_g2(out, &a);
    free(b);
    return 0;
}

int oracle_port_intt_coset_ntt(int log_n, uint8_t *data) {
    port_ntt *t = port_ntt_new(log_n);
    if (!t) return -1;
    port_intt_coset_ntt(t, (fp_t *)data);
    port_ntt_free(t);
    return 0;
}

/* A prepared port prover: the parsed key and the domain tables, built once
 * (the reference's warm mode: key parsed and tables cached before timing). */
typedef struct { const zkey_t *k; port_ntt *t; } port_prover;

void *oracle_port_prepare(const void *kv) {
    const zkey_t *k = kv;
    int log_n = 0;
    while (((size_t)1 << log_n) < k->domain_size) log_n++;
    port_prover *p = malloc(sizeof *p);
    p->k = k;
    p->t = port_ntt_new(log_n);
    if (!p->t) { free(p); return NULL; }
    return p;
}

void oracle_port_free(void *pv) {
    port_prover *p = pv;
    if (!p) return;
    port_ntt_free(p->t);
    free(p);
}

int oracle_port_prove(const void *pv, const uint8_t *w_mont, size_t n, const uint8_t *r_mont, const uint8_t *s_mont,
                      uint8_t *proof_out) {
    const port_prover *pp = pv;
    if (n != pp->k->n_vars) return -1;
    fp_t r, s;
    ld(&r, r_mont); ld(&s, s_mont);
    proof_t p;
    if (port_prove(pp->k, pp->t, (const fp_t *)w_mont, &r, &s, &p) != 0) return -1;
    pack_proof(proof_out, &p);
    return 0;
}

/* the fast product against the oracle's, for the CPU tests: which 0 = Fr, 1 = Fq */
void oracle_port_fp_mul(int which, const uint8_t *a, const uint8_t *b, uint8_t *out) {
    fp_t x, y, z;
    ld(&x, a); ld(&y, b);
    if (which) pq_mul(&z, &x, &y); else pr_mul(&z, &x, &y);
    st(out, &z);
}
void oracle_port_fq_inv(const uint8_t *a, uint8_t *out) {
    fp_t x, z;
    ld(&x, a);
    pq_inv(&z, &x);
    st(out, &z);
}
