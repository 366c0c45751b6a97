/*
 * CPU ORACLE -- test infrastructure only (see bn254.h).
 *
 * The timed CPU baseline: the reference CPU prover's algorithms restated for
 * speed (port_msm.c, port_ntt.c, port_prove.c), separate from the plain
 * restatement the tests check the CUDA product against (field.c ... groth16.c),
 * whose results it must equal.
 */
#ifndef G16_ORACLE_PORT_H
#define G16_ORACLE_PORT_H
#include "oracle.h"
#include "port_field.h"

#ifdef __cplusplus
extern "C" {
#endif

/* MSMs (crates/msm/src/lib.rs pippenger, portable path); scalars in standard form */
void port_msm_g1(g1j_t *out, const g1a_t *bases, const fp_t *scalars_std, size_t n);
void port_msm_g2(g2j_t *out, const g2a_t *bases, const fp_t *scalars_std, size_t n);
/* the same as tasks of an enclosing OpenMP parallel region */
void port_msm_g1_tasks(g1j_t *out, const g1a_t *bases, const fp_t *scalars_std, size_t n, int threads);
void port_msm_g2_tasks(g2j_t *out, const g2a_t *bases, const fp_t *scalars_std, size_t n, int threads);

/* crates/ntt/src/lib.rs intt_coset_ntt with 2^11-element cache blocks, as tasks */
typedef struct port_ntt port_ntt;
port_ntt *port_ntt_new(int log_n);
void port_ntt_free(port_ntt *t);
void port_intt_coset_ntt_tasks(const port_ntt *t, fp_t *a);
void port_intt_coset_ntt(const port_ntt *t, fp_t *a);

/* stages 0-11 (crates/groth16/src/cpu.rs h_and_msms + prove.rs assembly) */
int port_prove(const zkey_t *k, const port_ntt *t, const fp_t *w, const fp_t *r, const fp_t *s, proof_t *p);

#ifdef __cplusplus
}
#endif
#endif
