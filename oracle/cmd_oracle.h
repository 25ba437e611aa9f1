/*
 * cmd_oracle.h -- CPU restatement of the Classic McEliece decrypt path of
 * somesh-vas/CM_Decrypt_ (CPU/ tree).  TEST INFRASTRUCTURE ONLY: this code is
 * the checker for the CUDA engine.  Only tests/, the smoke entry point and the
 * CPU-baseline leg of bench.py may load it; the product never links it.
 *
 * Runtime-parameterised over the five parameter sets instead of the
 * reference's one-binary-per-set #defines (CPU/param/param<set>/include/common.h).
 * Each function names the reference lines whose behaviour it restates.
 */
#ifndef CMD_ORACLE_H
#define CMD_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int set_id;      /* 348864, 460896, 6688128, 6960119, 8192128 */
    int m;           /* GFBITS */
    int n;           /* SYS_N */
    int t;           /* SYS_T */
    int ct_bytes;    /* crypto_kem_CIPHERTEXTBYTES == SYND_BYTES */
    int sk_bytes;    /* crypto_kem_SECRETKEYBYTES */
    int sb;          /* 8 * SYND_BYTES: ciphertext bits fed to synd() */
    int cond_bytes;  /* Benes control bytes: 2^(m-4) * (2m-1) */
} o_params;

/* Fills *p for a set id; returns 0, or -4 (KAT_CRYPTO_FAILURE) if unknown. */
int o_params_get(int set_id, o_params *p);

/* GF(2^m) arithmetic (CPU/src/common/gf_13.c:86-111, 257-271;
 * CPU/param/param348864/src/gf.c:103-184). */
uint16_t o_gf_mul(int m, uint16_t a, uint16_t b);
uint16_t o_gf_inv(int m, uint16_t a);               /* a^(2^m-2); 0 -> 0 */
uint16_t o_gf_frac(int m, uint16_t den, uint16_t num); /* num/den */
uint16_t o_bitrev(int m, uint16_t a);

/* Bulk helpers so tests can sweep whole fields without per-call overhead. */
void o_gf_mul_row(int m, uint16_t a, uint16_t *out);   /* out[b] = a*b, b<2^m */
void o_gf_frac_row(int m, uint16_t num, uint16_t *out); /* out[d] = num/d */

/* Secret-key expansion (CPU/param/param6960119/src/util.c:60-100,
 * CPU/src/common/root_13.c:95-211).  g has t+1 entries (g[t]=1), L has n,
 * inv_tab has sb*2t entries, row-major [bit][power]. */
int o_support_gen(const o_params *p, const uint8_t *cond, uint16_t *L);
int o_key_expand(const o_params *p, const uint8_t *sk, uint16_t *g,
                 uint16_t *L, uint16_t *inv_tab);
uint16_t o_eval(int m, int t, const uint16_t *f, uint16_t a);

/* Per-ciphertext stages (util.c:102-114, bm.c:12-68, root_13.c:216-240). */
void o_synd(const o_params *p, const uint16_t *inv_tab, const uint8_t *ct,
            uint16_t *s);
void o_bm(const o_params *p, const uint16_t *s, uint16_t *locator);
void o_root(const o_params *p, const uint16_t *locator, const uint16_t *L,
            uint16_t *images);

/* Whole decrypt of `count` ciphertexts into n/8-byte error vectors
 * (CPU/param/param6960119/src/decrypt.c:163-177 + build_error_vector). */
int o_decrypt_batch(const o_params *p, const uint8_t *sk, const uint8_t *cts,
                    size_t count, uint8_t *err_bytes, int nthreads);

/* Errorstream text (decrypt.c:55-66): " %d" per set bit, then '\n'.
 * Returns the number of bytes written, or -1 if cap is too small. */
/* KEM decapsulation acceptance test (no counterpart in the reference; see the
 * definition): accept[c] = padding zero && wt(e_c) == t && the 2t syndromes
 * of e_c over all n support points equal those of ciphertext c. */
int o_decap_accept(const o_params *p, const uint8_t *sk, const uint8_t *cts,
                   const uint8_t *errs, size_t count, uint8_t *accept);

long o_errorstream_format(const o_params *p, const uint8_t *err_bytes,
                          size_t count, char *out, size_t cap);

/* Key generation stages of crypto_kem_keypair (kem/common/core/operations.c:
 * 36-107); the seed expansion around them is restated in oracle.py.
 *  o_kg_genpoly: minimal polynomial of f in GF((2^m)^t) (sk_gen.c:24-85 with
 *    kem/variant_<set>/gf.c GF_mul); irr gets its t low coefficients; -1 if
 *    the degree is below t.
 *  o_kg_pk_gen: public key (mt rows of (n-mt+7)/8 bytes) and support
 *    permutation pi (2^m entries) from the Goppa polynomial (t coefficients)
 *    and 2^m random words (pk_gen.c:29-149); -1 when the draw is rejected.
 *  o_kg_controlbits: Benes control bits of pi, (2m-1) 2^(m-4) bytes
 *    (controlbits.c:22-220). */
int o_kg_genpoly(const o_params *p, const uint16_t *f, uint16_t *irr);
int o_kg_pk_gen(const o_params *p, const uint16_t *irr, const uint32_t *perm,
                uint8_t *pk, int16_t *pi);
void o_kg_controlbits(int m, const int16_t *pi, uint8_t *out);


/* Test inputs for the reference-only bench arm and CPU tests.
 *  o_encrypt_batch: ciphertexts (ct_bytes each) of `count` error vectors
 *    (n/8 bytes each) under a public key, by encrypt.c:87-120's syndrome rule.
 *  o_random_errors: `count` error vectors of weight exactly t, uniform over
 *    [0, n), from a seeded stream. */
int o_encrypt_batch(const o_params *p, const uint8_t *pk, const uint8_t *errs,
                    size_t count, uint8_t *cts);
void o_random_errors(const o_params *p, uint64_t seed, size_t count,
                     uint8_t *errs);

#ifdef __cplusplus
}
#endif
#endif
