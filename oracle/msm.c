/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * Pippenger MSM restating crates/msm/src/lib.rs:
 *   - prescan (:534): scalar 0 and infinity bases dropped, scalar 1 folded
 *     into one running addition;
 *   - window_size (:160-172): the c in 3..=16 minimising
 *     ceil(255/c) * (m + 3 * 2^(c-1)) over the m general scalars;
 *   - signed_digit (:319-333): carry-free signed recoding over
 *     RECODE_BITS = 255 bits (:94), digits in [-2^(c-1), 2^(c-1)] and
 *     2^(c-1) buckets per window;
 *   - per-window, per-chunk bucket fill, running-sum reduction and Horner
 *     over the windows (:1684-1817).
 * Buckets are Jacobian here (XYZZ in the reference); the sum is a group
 * element, identical after affine normalisation either way.
 */
#include "oracle.h"
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define RECODE_BITS 255
#define MAX_WINDOW 16

int msm_window_size(size_t m) {
    int best = 3;
    unsigned __int128 best_cost = ~(unsigned __int128)0;
    for (int c = 3; c <= MAX_WINDOW; c++) {
        unsigned __int128 windows = (RECODE_BITS + c - 1) / c;
        unsigned __int128 cost = windows * ((unsigned __int128)m + 3 * ((unsigned __int128)1 << (c - 1)));
        if (cost < best_cost) { best_cost = cost; best = c; }
    }
    return best;
}

static uint64_t read_bits(const uint64_t *limbs, int off, int width) {
    int idx = off / 64;
    if (idx >= 4) return 0;
    int sh = off % 64;
    uint64_t buf = limbs[idx] >> sh;
    if (sh + width > 64 && idx + 1 < 4) buf |= limbs[idx + 1] << (64 - sh);
    return buf & ((1ULL << width) - 1);
}

static int signed_digit(const uint64_t *limbs, int w, int c) {
    int off = w * c;
    int64_t b = (int64_t)read_bits(limbs, off, c);
    int64_t d = b - ((b >> (c - 1)) << c);
    int64_t carry = off == 0 ? 0 : (int64_t)read_bits(limbs, off - 1, 1);
    return (int)(d + carry);
}

static int is_one_std(const fp_t *s) { return s->v[0] == 1 && !s->v[1] && !s->v[2] && !s->v[3]; }

static int n_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

#define DEFINE_MSM(G, FT)                                                                 \
void msm_##G(G##j_t *out, const G##a_t *bases, const fp_t *s, size_t n) {                  \
    G##j_t ones;                                                                           \
    G##j_set_inf(&ones);                                                                   \
    uint32_t *idx = malloc((n ? n : 1) * sizeof(uint32_t));                                \
    size_t m = 0;                                                                          \
    for (size_t i = 0; i < n; i++) {                                                       \
        if (bases[i].inf || fp_is_zero(&s[i])) continue;                                  \
        if (is_one_std(&s[i])) { G##j_add_affine(&ones, &ones, &bases[i]); continue; }     \
        idx[m++] = (uint32_t)i;                                                            \
    }                                                                                      \
    if (m == 0) { *out = ones; free(idx); return; }                                        \
    int c = msm_window_size(m);                                                            \
    int W = (RECODE_BITS + c - 1) / c;                                                     \
    size_t B = (size_t)1 << (c - 1);                                                       \
    int th = n_threads();                                                                  \
    size_t chunks = ((size_t)2 * th + W - 1) / W;                                          \
    size_t cap = m / (16 * B); if (cap < 1) cap = 1;                                       \
    if (chunks > cap) chunks = cap;                                                        \
    if (chunks < 1) chunks = 1;                                                            \
    size_t chunk_len = (m + chunks - 1) / chunks;                                          \
    G##j_t *part = malloc(sizeof(G##j_t) * W * chunks);                                    \
    long tasks = (long)(W * chunks);                                                       \
    _Pragma("omp parallel for schedule(dynamic, 1)")                                       \
    for (long t = 0; t < tasks; t++) {                                                     \
        int w = (int)(t / (long)chunks);                                                   \
        size_t ci = (size_t)(t % (long)chunks);                                            \
        size_t lo = ci * chunk_len, hi = lo + chunk_len < m ? lo + chunk_len : m;          \
        G##j_t *bk = malloc(sizeof(G##j_t) * B);                                           \
        for (size_t b = 0; b < B; b++) G##j_set_inf(&bk[b]);                               \
        for (size_t k = lo; k < hi; k++) {                                                 \
            uint32_t i = idx[k];                                                           \
            int d = signed_digit(s[i].v, w, c);                                            \
            if (d > 0) G##j_add_affine(&bk[d - 1], &bk[d - 1], &bases[i]);                 \
            else if (d < 0) {                                                              \
                G##a_t neg = bases[i];                                                     \
                G##j_t tmp; G##j_from_affine(&tmp, &neg); G##j_neg(&tmp, &tmp);            \
                G##a_t na; na.x = tmp.x; na.y = tmp.y; na.inf = 0;                         \
                G##j_add_affine(&bk[-d - 1], &bk[-d - 1], &na);                            \
            }                                                                              \
        }                                                                                  \
        G##j_t run, sum;                                                                   \
        G##j_set_inf(&run); G##j_set_inf(&sum);                                            \
        for (size_t b = B; b-- > 0;) {                                                     \
            G##j_add(&run, &run, &bk[b]);                                                  \
            G##j_add(&sum, &sum, &run);                                                    \
        }                                                                                  \
        part[t] = sum;                                                                     \
        free(bk);                                                                          \
    }                                                                                      \
    G##j_t acc;                                                                            \
    G##j_set_inf(&acc);                                                                    \
    for (int w = W - 1; w >= 0; w--) {                                                     \
        for (int k = 0; k < c && w != W - 1; k++) G##j_dbl(&acc, &acc);                    \
        for (size_t ci = 0; ci < chunks; ci++) G##j_add(&acc, &acc, &part[(size_t)w * chunks + ci]); \
    }                                                                                      \
    G##j_add(out, &acc, &ones);                                                            \
    free(part);                                                                            \
    free(idx);                                                                             \
}

DEFINE_MSM(g1, fp_t)
DEFINE_MSM(g2, fq2_t)
