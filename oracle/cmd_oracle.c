/*
 * cmd_oracle.c -- CPU restatement of the reference decrypt path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  Plain,
 * deliberately unoptimised C: every step is written the most direct way so it
 * can be read against the reference and against the CUDA engine.  Where the
 * reference uses a clever bitsliced formulation (the Benes network on 64x64
 * transposed words, the Itoh-Tsujii inversion chains) this file states the
 * same mathematical operation directly; tests pin the two against each other
 * on every golden key and on exhaustive field sweeps.
 */
#include "cmd_oracle.h"

#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* Parameter sets: CPU/param/param<set>/include/common.h:14-29 and
 * kem/variant_<set>/crypto_kem_mceliece<set>.h:4-6 (sk/ct sizes). */
int o_params_get(int set_id, o_params *p)
{
    int m, n, t, ct, sk;
    switch (set_id) {
    case 348864:  m = 12; n = 3488; t = 64;  ct = 96;  sk = 6492;  break;
    case 460896:  m = 13; n = 4608; t = 96;  ct = 156; sk = 13608; break;
    case 6688128: m = 13; n = 6688; t = 128; ct = 208; sk = 13932; break;
    case 6960119: m = 13; n = 6960; t = 119; ct = 194; sk = 13948; break;
    case 8192128: m = 13; n = 8192; t = 128; ct = 208; sk = 14120; break;
    default: return -4;
    }
    p->set_id = set_id;
    p->m = m;
    p->n = n;
    p->t = t;
    p->ct_bytes = ct;          /* == SYND_BYTES = ceil(m*t/8) */
    p->sk_bytes = sk;
    p->sb = 8 * ct;            /* sb = SYND_BYTES*8 (common.h:29) */
    p->cond_bytes = (1 << (m - 4)) * (2 * m - 1);
    return 0;
}

/* Field moduli: x^12+x^3+1 (CPU/param/param348864/src/gf.c:116-122) and
 * x^13+x^4+x^3+x+1 (CPU/src/common/gf_13.c:103-108). */
static uint32_t field_poly(int m) { return m == 12 ? 0x1009u : 0x201Bu; }

/* Schoolbook carry-less product followed by long division by the modulus;
 * the reference's two-fold reduction (gf_13.c:104-108) is the same map. */
uint16_t o_gf_mul(int m, uint16_t a, uint16_t b)
{
    uint32_t prod = 0;
    for (int i = 0; i < m; i++)
        if ((b >> i) & 1u)
            prod ^= (uint32_t)a << i;
    uint32_t poly = field_poly(m);
    for (int k = 2 * m - 2; k >= m; k--)
        if ((prod >> k) & 1u)
            prod ^= poly << (k - m);
    return (uint16_t)(prod & ((1u << m) - 1u));
}

/* a^(2^m-2) by plain square-and-multiply.  gf_13.c:257-271 and
 * param348864/src/gf.c:150-184 compute the same power with addition chains;
 * both send 0 to 0, which the syndrome table and BM rely on. */
uint16_t o_gf_inv(int m, uint16_t a)
{
    uint32_t e = (1u << m) - 2u;
    uint16_t result = 1, base = a;
    while (e) {
        if (e & 1u)
            result = o_gf_mul(m, result, base);
        base = o_gf_mul(m, base, base);
        e >>= 1;
    }
    return result;
}

/* gf_frac(den, num) = num/den (gf_13.c:257-271; param348864/src/gf.c:181-184). */
uint16_t o_gf_frac(int m, uint16_t den, uint16_t num)
{
    return o_gf_mul(m, o_gf_inv(m, den), num);
}

/* m-bit reversal (gf_13.c:8-16 reverses 16 bits then drops 3; m=12 drops 4). */
uint16_t o_bitrev(int m, uint16_t a)
{
    uint16_t r = 0;
    for (int i = 0; i < m; i++)
        if ((a >> i) & 1u)
            r |= (uint16_t)(1u << (m - 1 - i));
    return r;
}

void o_gf_mul_row(int m, uint16_t a, uint16_t *out)
{
    for (uint32_t b = 0; b < (1u << m); b++)
        out[b] = o_gf_mul(m, a, (uint16_t)b);
}

void o_gf_frac_row(int m, uint16_t num, uint16_t *out)
{
    for (uint32_t d = 0; d < (1u << m); d++)
        out[d] = o_gf_frac(m, (uint16_t)d, num);
}

/* Support generation (root_13.c:181-211 with apply_benes at :95-177;
 * m=12: param348864/src/root.c:67-199).
 *
 * The reference permutes m bit-planes of the table bitrev(0..2^m-1) through a
 * (2m-1)-layer Benes network.  Stated element-wise: layer l swaps entries p
 * and p + 2^e (bit e of p clear) where e = l for l < m and e = 2m-2-l after,
 * and the swap is taken when control bit number l*2^(m-1) + q is set, q being
 * p with bit e deleted; control bits are numbered little-endian within
 * bytes.  The support is the first n entries of the permuted table. */
int o_support_gen(const o_params *p, const uint8_t *cond, uint16_t *L)
{
    const int m = p->m;
    const uint32_t size = 1u << m;
    uint16_t *v = (uint16_t *)malloc(size * sizeof(uint16_t));
    if (!v)
        return -1;
    for (uint32_t i = 0; i < size; i++)
        v[i] = o_bitrev(m, (uint16_t)i);
    for (int layer = 0; layer < 2 * m - 1; layer++) {
        const int e = layer < m ? layer : 2 * m - 2 - layer;
        const uint32_t stride = 1u << e;
        const uint32_t base = (uint32_t)layer << (m - 1);
        for (uint32_t pos = 0; pos < size; pos++) {
            if (pos & stride)
                continue;
            uint32_t q = ((pos >> (e + 1)) << e) | (pos & (stride - 1));
            uint32_t bit = base + q;
            if ((cond[bit >> 3] >> (bit & 7)) & 1u) {
                uint16_t tmp = v[pos];
                v[pos] = v[pos + stride];
                v[pos + stride] = tmp;
            }
        }
    }
    memcpy(L, v, (size_t)p->n * sizeof(uint16_t));
    free(v);
    return 0;
}

/* Horner evaluation, f of degree t (root_13.c:216-230). */
uint16_t o_eval(int m, int t, const uint16_t *f, uint16_t a)
{
    uint16_t r = f[t];
    for (int i = t - 1; i >= 0; i--)
        r = (uint16_t)(o_gf_mul(m, r, a) ^ f[i]);
    return r;
}

/* sk = [32 B seed][8 B pivots][t LE u16 Goppa coefficients][Benes bits][s]
 * (util.c:60-72: prefix 40, coefficients masked to m bits, g[t] = 1), then
 * inv_tab[b][j] = L_b^j / g(L_b)^2 for b < sb, j < 2t (util.c:86-100). */
int o_key_expand(const o_params *p, const uint8_t *sk, uint16_t *g,
                 uint16_t *L, uint16_t *inv_tab)
{
    const int m = p->m, t = p->t;
    const uint16_t mask = (uint16_t)((1u << m) - 1u);
    const uint8_t *q = sk + 40;
    for (int i = 0; i < t; i++)
        g[i] = (uint16_t)((q[2 * i] | (q[2 * i + 1] << 8)) & mask);
    g[t] = 1;
    if (o_support_gen(p, sk + 40 + 2 * t, L) != 0)
        return -1;
    if (inv_tab) {
        for (int b = 0; b < p->sb; b++) {
            uint16_t v = o_eval(m, t, g, L[b]);
            uint16_t inv = o_gf_inv(m, o_gf_mul(m, v, v));
            uint16_t *row = inv_tab + (size_t)b * 2 * t;
            row[0] = inv;
            for (int j = 1; j < 2 * t; j++)
                row[j] = o_gf_mul(m, row[j - 1], L[b]);
        }
    }
    return 0;
}

/* s_j = XOR of inv_tab[b][j] over set ciphertext bits b < sb (util.c:102-114;
 * the caller copies SYND_BYTES of ct, decrypt.c:163-164). */
void o_synd(const o_params *p, const uint16_t *inv_tab, const uint8_t *ct,
            uint16_t *s)
{
    const int t2 = 2 * p->t;
    memset(s, 0, (size_t)t2 * sizeof(uint16_t));
    for (int b = 0; b < p->sb; b++) {
        if (!((ct[b >> 3] >> (b & 7)) & 1u))
            continue;
        const uint16_t *row = inv_tab + (size_t)b * t2;
        for (int j = 0; j < t2; j++)
            s[j] ^= row[j];
    }
}

/* Berlekamp-Massey exactly as CPU/src/common/bm.c:12-68: C and B hold t+1
 * coefficients, the discrepancy sums i <= min(N,t), B <- x*B drops B[t], and
 * the output is reversed, out[i] = C[t-i]. */
void o_bm(const o_params *p, const uint16_t *s, uint16_t *locator)
{
    const int m = p->m, t = p->t;
    uint16_t C[130], B[130], Tmp[130];
    uint16_t b = 1;
    int L = 0;
    for (int i = 0; i <= t; i++)
        C[i] = B[i] = 0;
    C[0] = 1;
    B[1] = 1;
    for (int N = 0; N < 2 * t; N++) {
        uint16_t d = 0;
        int lim = N < t ? N : t;
        for (int i = 0; i <= lim; i++)
            d ^= o_gf_mul(m, C[i], s[N - i]);
        int nonzero = d != 0;
        int lengthen = nonzero && (N >= 2 * L);
        memcpy(Tmp, C, (size_t)(t + 1) * sizeof(uint16_t));
        uint16_t f = o_gf_frac(m, b, d);
        if (nonzero)
            for (int i = 0; i <= t; i++)
                C[i] ^= o_gf_mul(m, f, B[i]);
        if (lengthen) {
            L = N + 1 - L;
            memcpy(B, Tmp, (size_t)(t + 1) * sizeof(uint16_t));
            b = d;
        }
        for (int i = t; i >= 1; i--)
            B[i] = B[i - 1];
        B[0] = 0;
    }
    for (int i = 0; i <= t; i++)
        locator[i] = C[t - i];
}

/* images[i] = locator evaluated at L[i], i < n (root_13.c:233-240). */
void o_root(const o_params *p, const uint16_t *locator, const uint16_t *L,
            uint16_t *images)
{
    for (int i = 0; i < p->n; i++)
        images[i] = o_eval(p->m, p->t, locator, L[i]);
}

typedef struct {
    const o_params *p;
    const uint16_t *inv_tab;
    const uint16_t *L;
    const uint8_t *cts;
    uint8_t *err;
    size_t begin, end;
} o_job;

static void *o_worker(void *arg)
{
    o_job *job = (o_job *)arg;
    const o_params *p = job->p;
    uint16_t s[256], loc[130];
    uint16_t *images = (uint16_t *)malloc((size_t)p->n * sizeof(uint16_t));
    if (!images)
        return (void *)1;
    for (size_t c = job->begin; c < job->end; c++) {
        o_synd(p, job->inv_tab, job->cts + c * (size_t)p->ct_bytes, s);
        o_bm(p, s, loc);
        o_root(p, loc, job->L, images);
        /* build_error_vector (decrypt.c:43-53): bit i set iff image == 0. */
        uint8_t *e = job->err + c * (size_t)(p->n / 8);
        memset(e, 0, (size_t)(p->n / 8));
        for (int i = 0; i < p->n; i++)
            if (images[i] == 0)
                e[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
    free(images);
    return NULL;
}

int o_decrypt_batch(const o_params *p, const uint8_t *sk, const uint8_t *cts,
                    size_t count, uint8_t *err_bytes, int nthreads)
{
    uint16_t g[130];
    uint16_t *L = (uint16_t *)malloc((size_t)p->n * sizeof(uint16_t));
    uint16_t *tab = (uint16_t *)malloc((size_t)p->sb * 2 * p->t * sizeof(uint16_t));
    int rc = 0;
    if (!L || !tab) {
        rc = -1;
        goto out;
    }
    if (o_key_expand(p, sk, g, L, tab) != 0) {
        rc = -1;
        goto out;
    }
    if (nthreads < 1)
        nthreads = 1;
    if ((size_t)nthreads > count)
        nthreads = count ? (int)count : 1;
    {
        pthread_t th[256];
        o_job jobs[256];
        if (nthreads > 256)
            nthreads = 256;
        size_t per = (count + (size_t)nthreads - 1) / (size_t)nthreads;
        for (int i = 0; i < nthreads; i++) {
            jobs[i].p = p;
            jobs[i].inv_tab = tab;
            jobs[i].L = L;
            jobs[i].cts = cts;
            jobs[i].err = err_bytes;
            jobs[i].begin = (size_t)i * per < count ? (size_t)i * per : count;
            jobs[i].end = jobs[i].begin + per < count ? jobs[i].begin + per : count;
            if (nthreads == 1) {
                if (o_worker(&jobs[0]))
                    rc = -1;
            } else if (pthread_create(&th[i], NULL, o_worker, &jobs[i]) != 0) {
                rc = -1;
                nthreads = i;
                break;
            }
        }
        if (nthreads > 1)
            for (int i = 0; i < nthreads; i++) {
                void *ret = NULL;
                pthread_join(th[i], &ret);
                if (ret)
                    rc = -1;
            }
    }
out:
    free(L);
    free(tab);
    return rc;
}

long o_errorstream_format(const o_params *p, const uint8_t *err_bytes,
                          size_t count, char *out, size_t cap)
{
    size_t pos = 0;
    char buf[16];
    for (size_t c = 0; c < count; c++) {
        const uint8_t *e = err_bytes + c * (size_t)(p->n / 8);
        for (int i = 0; i < p->n; i++) {
            if (!((e[i >> 3] >> (i & 7)) & 1u))
                continue;
            int len = snprintf(buf, sizeof buf, " %d", i);
            if (pos + (size_t)len > cap)
                return -1;
            memcpy(out + pos, buf, (size_t)len);
            pos += (size_t)len;
        }
        if (pos + 1 > cap)
            return -1;
        out[pos++] = '\n';
    }
    return (long)pos;
}

/* KEM decapsulation check.  No counterpart in the reference (it encapsulates
 * only: kem/common/core/operations.c:15-34 hashes K = SHAKE256(1 || e || C));
 * this is the Classic McEliece decapsulation's acceptance test, stated with
 * the reference's own syndrome: accept[c] = 1 iff the padding bits mt..sb-1
 * of ciphertext c are zero, e_c has weight exactly t, and the 2t syndromes
 * of e_c over all n support points (sum over set bits i of L_i^j / g(L_i)^2)
 * equal the syndromes of the ciphertext (o_synd), i.e. the received word
 * plus e_c is a codeword.  The session key is then SHAKE256(b || v || C),
 * v = e (b = 1) or the sk's random string s (b = 0). */
int o_decap_accept(const o_params *p, const uint8_t *sk, const uint8_t *cts,
                   const uint8_t *errs, size_t count, uint8_t *accept)
{
    const int m = p->m, t = p->t, t2 = 2 * p->t, mt = m * t;
    uint16_t g[130];
    uint16_t *L = (uint16_t *)malloc((size_t)p->n * sizeof(uint16_t));
    uint16_t *tab = (uint16_t *)malloc((size_t)p->sb * t2 * sizeof(uint16_t));
    uint16_t *ginv2 = (uint16_t *)malloc((size_t)p->n * sizeof(uint16_t));
    int rc = 0;
    if (!L || !tab || !ginv2 || o_key_expand(p, sk, g, L, tab) != 0) {
        rc = -1;
        goto out;
    }
    for (int i = 0; i < p->n; i++) {
        uint16_t v = o_eval(m, t, g, L[i]);
        ginv2[i] = o_gf_inv(m, o_gf_mul(m, v, v));
    }
    for (size_t c = 0; c < count; c++) {
        const uint8_t *ct = cts + c * (size_t)p->ct_bytes;
        const uint8_t *e = errs + c * (size_t)(p->n / 8);
        int ok = 1;
        for (int b = mt; b < p->sb; b++)
            if ((ct[b >> 3] >> (b & 7)) & 1u)
                ok = 0;
        uint16_t s[256], se[256];
        o_synd(p, tab, ct, s);
        memset(se, 0, sizeof se);
        int w = 0;
        for (int i = 0; i < p->n; i++) {
            if (!((e[i >> 3] >> (i & 7)) & 1u))
                continue;
            w++;
            uint16_t x = ginv2[i];
            for (int j = 0; j < t2; j++) {
                se[j] ^= x;
                x = o_gf_mul(m, x, L[i]);
            }
        }
        if (w != t)
            ok = 0;
        for (int j = 0; j < t2; j++)
            if (s[j] != se[j])
                ok = 0;
        accept[c] = (uint8_t)ok;
    }
out:
    free(L);
    free(tab);
    free(ginv2);
    return rc;
}
