/*
 * ref_harness.c -- thin C driver around the reference's own CPU decoder
 * sources (somesh-vas/CM_Decrypt_ CPU/), compiled once per parameter set by
 * oracle/Makefile into oracle/_ref/libref_<set>.so.  TEST INFRASTRUCTURE ONLY.
 *
 * It defines the globals that CPU/param/param<set>/src/util.c declares extern
 * (L, g, e_inv, inverse_elements; see e.g. CPU/param/param6960119/src/
 * decrypt.c:93-98), parses the secret key the way util.c:60-72 does, and then
 * calls the reference's support_gen / compute_inverses / synd / bm / root
 * unchanged.  Nothing here re-implements the algorithm.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "common.h"
#include "gf.h"
#include "bm.h"
#include "root.h"

#define API __attribute__((visibility("default")))

gf L[SYS_N];
gf g[SYS_T + 1];
gf e_inv[SYS_N];
gf inverse_elements[sb][2 * SYS_T];

API int ref_info(int *out6)
{
    out6[0] = GFBITS;
    out6[1] = SYS_N;
    out6[2] = SYS_T;
    out6[3] = crypto_kem_CIPHERTEXTBYTES;
    out6[4] = crypto_kem_SECRETKEYBYTES;
    out6[5] = sb;
    return 0;
}

/* util.c:60-72: g from sk+40 (t LE coefficients), g[t] = 1, support from the
 * Benes bits that follow; then util.c:86-100 builds the inverse table. */
API int ref_load_sk(const unsigned char *sk)
{
    const unsigned char *q = sk + 40;
    for (int i = 0; i < SYS_T; i++) {
        g[i] = load_gf(q);
        q += 2;
    }
    g[SYS_T] = 1;
    support_gen(L, q);
    compute_inverses();
    return 0;
}

API void ref_get_support(uint16_t *out) { memcpy(out, L, sizeof L); }
API void ref_get_goppa(uint16_t *out) { memcpy(out, g, sizeof g); }
API void ref_get_inverse_table(uint16_t *out)
{
    memcpy(out, inverse_elements, sizeof inverse_elements);
}

/* decrypt.c:163-164: SYND_BYTES of the ciphertext, zero tail, then synd(). */
API void ref_synd(const unsigned char *ct, uint16_t *s)
{
    unsigned char r[SYS_N / 8];
    memcpy(r, ct, SYND_BYTES);
    memset(r + SYND_BYTES, 0, sizeof r - SYND_BYTES);
    synd(s, r);
}

API void ref_bm(const uint16_t *s, uint16_t *locator)
{
    gf tmp[2 * SYS_T];
    memcpy(tmp, s, sizeof tmp);
    bm(locator, tmp);
}

API void ref_root(const uint16_t *locator, uint16_t *images)
{
    gf f[SYS_T + 1];
    memcpy(f, locator, sizeof f);
    root(images, f, L);
}

API uint16_t ref_gf_mul(uint16_t a, uint16_t b) { return gf_mul(a, b); }
API uint16_t ref_gf_frac(uint16_t den, uint16_t num) { return gf_frac(den, num); }
API uint16_t ref_gf_inv(uint16_t a) { return gf_inv(a); }
API uint16_t ref_bitrev(uint16_t a) { return bitrev(a); }

API void ref_gf_mul_row(uint16_t a, uint16_t *out)
{
    for (uint32_t b = 0; b < (1u << GFBITS); b++)
        out[b] = gf_mul(a, (gf)b);
}

API void ref_gf_frac_row(uint16_t num, uint16_t *out)
{
    for (uint32_t d = 0; d < (1u << GFBITS); d++)
        out[d] = gf_frac((gf)d, num);
}

API void ref_support_from_cond(const unsigned char *cond, uint16_t *out)
{
    gf tmp[SYS_N];
    support_gen(tmp, cond);
    memcpy(out, tmp, sizeof tmp);
}

typedef struct {
    const unsigned char *cts;
    unsigned char *err;
    size_t begin, end;
} job_t;

/* The per-ciphertext loop of decrypt.c:163-177 plus build_error_vector
 * (decrypt.c:43-53); synd/bm/root only read the globals set above. */
static void *worker(void *arg)
{
    job_t *job = (job_t *)arg;
    unsigned char r[SYS_N / 8];
    gf s[2 * SYS_T], loc[SYS_T + 1];
    gf *images = (gf *)malloc(sizeof(gf) * SYS_N);
    if (!images)
        return (void *)1;
    for (size_t c = job->begin; c < job->end; c++) {
        memcpy(r, job->cts + c * crypto_kem_CIPHERTEXTBYTES, SYND_BYTES);
        memset(r + SYND_BYTES, 0, sizeof r - SYND_BYTES);
        synd(s, r);
        bm(loc, s);
        root(images, loc, L);
        unsigned char *e = job->err + c * (SYS_N / 8);
        memset(e, 0, SYS_N / 8);
        for (int i = 0; i < SYS_N; i++)
            if (images[i] == 0)
                e[i >> 3] |= (unsigned char)(1u << (i & 7));
    }
    free(images);
    return NULL;
}

API int ref_decrypt_batch(const unsigned char *cts, size_t count,
                          unsigned char *err, int nthreads)
{
    pthread_t th[256];
    job_t jobs[256];
    int rc = 0;
    if (nthreads < 1)
        nthreads = 1;
    if (nthreads > 256)
        nthreads = 256;
    if ((size_t)nthreads > count)
        nthreads = count ? (int)count : 1;
    size_t per = (count + (size_t)nthreads - 1) / (size_t)nthreads;
    for (int i = 0; i < nthreads; i++) {
        jobs[i].cts = cts;
        jobs[i].err = err;
        jobs[i].begin = (size_t)i * per < count ? (size_t)i * per : count;
        jobs[i].end = jobs[i].begin + per < count ? jobs[i].begin + per : count;
    }
    if (nthreads == 1)
        return worker(&jobs[0]) ? -1 : 0;
    int started = 0;
    for (; started < nthreads; started++)
        if (pthread_create(&th[started], NULL, worker, &jobs[started]) != 0) {
            rc = -1;
            break;
        }
    for (int i = 0; i < started; i++) {
        void *ret = NULL;
        pthread_join(th[i], &ret);
        if (ret)
            rc = -1;
    }
    return rc;
}
