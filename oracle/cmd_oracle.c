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

/* ---- key generation ---------------------------------------------------- */

/* Reduction terms of the degree-t field polynomial F(y) defining GF((2^m)^t)
 * (kem/variant_<set>/gf.c GF_mul): y^t = sum of coef * y^off.
 *   348864: y^64 = y^3 + y + z      (z = the field element 2)
 *   460896: y^96 = y^10 + y^9 + y^6 + 1
 *   6688128, 8192128: y^128 = y^7 + y^2 + y + 1
 *   6960119: y^119 = y^8 + 1 */
static int ext_terms(int set_id, int *off, uint16_t *coef)
{
    switch (set_id) {
    case 348864: off[0] = 3; off[1] = 1; off[2] = 0; coef[0] = 1; coef[1] = 1; coef[2] = 2; return 3;
    case 460896: off[0] = 10; off[1] = 9; off[2] = 6; off[3] = 0; break;
    case 6960119: off[0] = 8; off[1] = 0; coef[0] = coef[1] = 1; return 2;
    default: off[0] = 7; off[1] = 2; off[2] = 1; off[3] = 0; break;
    }
    coef[0] = coef[1] = coef[2] = coef[3] = 1;
    return 4;
}

/* out = a * b in GF((2^m)^t): schoolbook product, then y^k (k >= t) folded
 * down from the top with the terms of F. */
static void ext_mul(const o_params *p, uint16_t *out, const uint16_t *a, const uint16_t *b)
{
    const int t = p->t, m = p->m;
    uint16_t prod[2 * 128];
    int off[4];
    uint16_t coef[4];
    const int nt = ext_terms(p->set_id, off, coef);
    memset(prod, 0, sizeof prod);
    for (int i = 0; i < t; i++)
        for (int j = 0; j < t; j++)
            prod[i + j] ^= o_gf_mul(m, a[i], b[j]);
    for (int k = 2 * t - 2; k >= t; k--)
        for (int u = 0; u < nt; u++)
            prod[k - t + off[u]] ^= coef[u] == 1 ? prod[k] : o_gf_mul(m, prod[k], coef[u]);
    memcpy(out, prod, (size_t)t * sizeof(uint16_t));
}

/* The minimal polynomial y^t + sum_{j<t} g_j y^j of f satisfies
 * f^t = sum_j g_j f^j: solve that t x t system over GF(2^m) (columns f^j) by
 * Gauss-Jordan elimination.  A singular system means f lies in a proper
 * subfield (degree below t): the reference rejects the draw (sk_gen.c:60-63). */
int o_kg_genpoly(const o_params *p, const uint16_t *f, uint16_t *irr)
{
    const int t = p->t, m = p->m;
    /* a[r][c]: row r = coordinate, column c = power f^c; column t = f^t */
    uint16_t *a = (uint16_t *)calloc((size_t)t * (t + 1), sizeof(uint16_t));
    uint16_t *pw = (uint16_t *)calloc((size_t)t, sizeof(uint16_t));
    uint16_t *nx = (uint16_t *)calloc((size_t)t, sizeof(uint16_t));
    if (!a || !pw || !nx) {
        free(a), free(pw), free(nx);
        return -2;
    }
#define A_(r, c) a[(size_t)(r) * (t + 1) + (c)]
    pw[0] = 1;
    for (int c = 0; c <= t; c++) {
        for (int r = 0; r < t; r++)
            A_(r, c) = pw[r];
        if (c < t) {
            ext_mul(p, nx, pw, f);
            memcpy(pw, nx, (size_t)t * sizeof(uint16_t));
        }
    }
    int rc = 0;
    for (int col = 0; col < t && rc == 0; col++) {
        int piv = -1;
        for (int r = col; r < t; r++)
            if (A_(r, col)) {
                piv = r;
                break;
            }
        if (piv < 0) {
            rc = -1;
            break;
        }
        if (piv != col)
            for (int c = 0; c <= t; c++) {
                uint16_t x = A_(piv, c);
                A_(piv, c) = A_(col, c);
                A_(col, c) = x;
            }
        const uint16_t inv = o_gf_inv(m, A_(col, col));
        for (int c = col; c <= t; c++)
            A_(col, c) = o_gf_mul(m, A_(col, c), inv);
        for (int r = 0; r < t; r++) {
            const uint16_t k = A_(r, col);
            if (r == col || !k)
                continue;
            for (int c = col; c <= t; c++)
                A_(r, c) ^= o_gf_mul(m, A_(col, c), k);
        }
    }
    if (rc == 0)
        for (int r = 0; r < t; r++)
            irr[r] = A_(r, t);
#undef A_
    free(a), free(pw), free(nx);
    return rc;
}

static int cmp_u64(const void *x, const void *y)
{
    const uint64_t a = *(const uint64_t *)x, b = *(const uint64_t *)y;
    return a < b ? -1 : a > b;
}

/* Support and parity-check matrix as in pk_gen.c:52-113: pi lists the
 * indices 0..2^m-1 ordered by their random word (rejected if two words are
 * equal), L_i = bitrev(pi_i), and row j*m + k, column i holds bit k of
 * L_i^j / g(L_i).  Gauss-Jordan elimination on the first mt columns must find
 * every pivot (else rejected); the reduced matrix is [I | T] whatever order
 * the eliminations take, and the public key is each row's bytes from byte
 * mt/8 on (pk_gen.c:145-146), so for mt not a multiple of 8 the first byte of
 * a row also carries the last mt mod 8 identity columns. */
int o_kg_pk_gen(const o_params *p, const uint16_t *irr, const uint32_t *perm, uint8_t *pk, int16_t *pi)
{
    const int m = p->m, n = p->n, t = p->t, mt = m * t, q = 1 << m;
    const int row_words = (n + 63) / 64, nbytes = n / 8, pk_row = (n - mt + 7) / 8;
    uint64_t *buf = (uint64_t *)malloc((size_t)q * sizeof(uint64_t));
    uint64_t *mat = (uint64_t *)calloc((size_t)mt * row_words, sizeof(uint64_t));
    uint16_t *g = (uint16_t *)malloc((size_t)(t + 1) * sizeof(uint16_t));
    uint16_t *L = (uint16_t *)malloc((size_t)n * sizeof(uint16_t));
    uint16_t *v = (uint16_t *)malloc((size_t)n * sizeof(uint16_t));
    int rc = 0;
    if (!buf || !mat || !g || !L || !v) {
        rc = -2;
        goto out;
    }
    for (int i = 0; i < q; i++)
        buf[i] = ((uint64_t)perm[i] << 31) | (uint64_t)i;
    qsort(buf, (size_t)q, sizeof(uint64_t), cmp_u64);
    for (int i = 1; i < q; i++)
        if ((buf[i - 1] >> 31) == (buf[i] >> 31)) {
            rc = -1;
            goto out;
        }
    for (int i = 0; i < q; i++)
        pi[i] = (int16_t)(buf[i] & (uint64_t)(q - 1));
    for (int i = 0; i < n; i++)
        L[i] = o_bitrev(m, (uint16_t)pi[i]);
    memcpy(g, irr, (size_t)t * sizeof(uint16_t));
    g[t] = 1;
    for (int i = 0; i < n; i++)
        v[i] = o_gf_inv(m, o_eval(m, t, g, L[i]));
    for (int j = 0; j < t; j++) {
        for (int i = 0; i < n; i++) {
            for (int k = 0; k < m; k++)
                if ((v[i] >> k) & 1u)
                    mat[(size_t)(j * m + k) * row_words + i / 64] |= 1ull << (i % 64);
            v[i] = o_gf_mul(m, v[i], L[i]);
        }
    }
    for (int c = 0; c < mt; c++) {
        const int w = c / 64;
        const uint64_t bit = 1ull << (c % 64);
        int piv = -1;
        for (int r = c; r < mt; r++)
            if (mat[(size_t)r * row_words + w] & bit) {
                piv = r;
                break;
            }
        if (piv < 0) {
            rc = -1;
            goto out;
        }
        uint64_t *pr = mat + (size_t)piv * row_words, *cr = mat + (size_t)c * row_words;
        if (piv != c)
            for (int x = 0; x < row_words; x++) {
                const uint64_t tmp = pr[x];
                pr[x] = cr[x];
                cr[x] = tmp;
            }
        for (int r = 0; r < mt; r++) {
            uint64_t *rr = mat + (size_t)r * row_words;
            if (r != c && (rr[w] & bit))
                for (int x = w; x < row_words; x++)
                    rr[x] ^= cr[x];
        }
    }
    for (int r = 0; r < mt; r++) {
        const uint64_t *rr = mat + (size_t)r * row_words;
        for (int b = 0; b < pk_row; b++) {
            const int byte = mt / 8 + b;
            pk[(size_t)r * pk_row + b] = byte < nbytes ? (uint8_t)(rr[byte / 8] >> (8 * (byte % 8))) : 0;
        }
    }
out:
    free(buf), free(mat), free(g), free(L), free(v);
    return rc;
}

/* Benes control bits by the cycle-labelling recursion of Nassimi and Sahni
 * in the formulation of Bernstein, "Verified fast formulas for control bits
 * for permutation networks" (2020), which controlbits.c:22-170 implements
 * with constant-time sorts; here every sort is the permutation algebra it
 * performs (inverses, compositions, gathers).  For pi on n = 2^w points:
 *   pibar(y) = pi(pi^-1(y ^ 1) ^ 1);  c(x) = min(x, pibar(x)); p = pibar^2;
 *   w-2 times: c <- min(c, c o p), p <- p o p;
 *   first-layer bit j = c(2j) & 1 (F swaps pair j when set);
 *   last-layer bit k = F(pi(2k)) & 1 (L swaps pair k when set);
 *   M = F o pi o L; the two halves q0(j) = M(2j)/2, q1(j) = M(2j+1)/2 recurse
 *   as the inner networks, interleaved at stride 2 step. */
static void cb_rec(uint8_t *out, long pos, long step, const int16_t *pi, int w, long n, int32_t *ws)
{
    if (w == 1) {
        out[pos >> 3] ^= (uint8_t)((pi[0] & 1) << (pos & 7));
        return;
    }
    int32_t *inv = ws, *pb = ws + n, *c = ws + 2 * n, *pp = ws + 3 * n, *tmp = ws + 4 * n, *F = ws + 5 * n;
    int16_t *q = (int16_t *)(ws + 6 * n);
    int32_t *rest = ws + 7 * n;
    for (long x = 0; x < n; x++)
        inv[pi[x]] = (int32_t)x;
    for (long y = 0; y < n; y++)
        pb[y] = pi[inv[y ^ 1] ^ 1];
    for (long x = 0; x < n; x++) {
        c[x] = x < pb[x] ? (int32_t)x : pb[x];
        pp[x] = pb[pb[x]];
    }
    for (int i = 1; i < w - 1; i++) {
        for (long x = 0; x < n; x++) {
            const int32_t cp = c[pp[x]];
            tmp[x] = cp < c[x] ? cp : c[x];
        }
        memcpy(c, tmp, (size_t)n * sizeof(int32_t));
        for (long x = 0; x < n; x++)
            tmp[x] = pp[pp[x]];
        memcpy(pp, tmp, (size_t)n * sizeof(int32_t));
    }
    for (long j = 0; j < n / 2; j++) {
        const int32_t fj = c[2 * j] & 1;
        out[(pos + j * step) >> 3] ^= (uint8_t)(fj << ((pos + j * step) & 7));
        F[2 * j] = (int32_t)(2 * j) + fj;
        F[2 * j + 1] = F[2 * j] ^ 1;
    }
    const long last = pos + (2 * w - 2) * step * (n / 2);
    for (long k = 0; k < n / 2; k++) {
        const int32_t a0 = F[pi[2 * k]], a1 = F[pi[2 * k + 1]];
        const int32_t lk = a0 & 1;
        out[(last + k * step) >> 3] ^= (uint8_t)(lk << ((last + k * step) & 7));
        /* M(L(y)) = F(pi(y)); L swaps the pair when lk is set */
        tmp[2 * k + lk] = a0;
        tmp[(2 * k + lk) ^ 1] = a1;
    }
    for (long j = 0; j < n / 2; j++) {
        q[j] = (int16_t)(tmp[2 * j] >> 1);
        q[j + n / 2] = (int16_t)(tmp[2 * j + 1] >> 1);
    }
    cb_rec(out, pos + (n / 2) * step, step * 2, q, w - 1, n / 2, rest);
    cb_rec(out, pos + (n / 2) * step + step, step * 2, q + n / 2, w - 1, n / 2, rest);
}

void o_kg_controlbits(int m, const int16_t *pi, uint8_t *out)
{
    const long n = 1L << m;
    memset(out, 0, (size_t)((2 * m - 1) * n / 2 + 7) / 8);
    /* each level takes 6.5 n int32 of workspace (q: n int16) */
    int32_t *ws = (int32_t *)malloc((size_t)(8 * n) * sizeof(int32_t) * 2);
    if (!ws)
        return;
    cb_rec(out, 0, 1, pi, m, n, ws);
    free(ws);
}

/* Niederreiter encryption of given error vectors with a public key: the
 * syndrome rule of kem/common/core/encrypt.c:87-120, where row i of H is the
 * pk row i placed in the last (n-mt+7)/8 bytes of an n-bit row with identity
 * bit i set, and ciphertext bit i = <row i, e>.  Computed column-wise: the
 * ciphertext is the XOR of the columns of H at the set bits of e. */
int o_encrypt_batch(const o_params *p, const uint8_t *pk, const uint8_t *errs, size_t count, uint8_t *cts)
{
    const int m = p->m, n = p->n, mt = m * p->t, nbytes = n / 8, row_b = (n - mt + 7) / 8;
    const int first = 8 * (nbytes - row_b), cb = p->ct_bytes;
    uint8_t *cols = (uint8_t *)calloc((size_t)(n - first) * (size_t)cb, 1);
    if (!cols)
        return -1;
    for (int i = 0; i < mt; i++) {
        const uint8_t *row = pk + (size_t)i * row_b;
        for (int j = first; j < n; j++) {
            const int b = j - first;
            int bit = (row[b >> 3] >> (b & 7)) & 1;
            if (j == i)
                bit = 1;
            if (bit)
                cols[(size_t)(j - first) * cb + (i >> 3)] |= (uint8_t)(1u << (i & 7));
        }
    }
    for (size_t c = 0; c < count; c++) {
        const uint8_t *e = errs + c * (size_t)nbytes;
        uint8_t *ct = cts + c * (size_t)cb;
        memset(ct, 0, (size_t)cb);
        for (int j = 0; j < n; j++) {
            if (!((e[j >> 3] >> (j & 7)) & 1))
                continue;
            if (j >= first) {
                const uint8_t *col = cols + (size_t)(j - first) * cb;
                for (int b = 0; b < cb; b++)
                    ct[b] ^= col[b];
            } else if (j < mt) {
                ct[j >> 3] ^= (uint8_t)(1u << (j & 7));
            }
        }
    }
    free(cols);
    return 0;
}

static uint64_t o_splitmix(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Error vectors of weight exactly t, uniform over [0, n): a partial
 * Fisher-Yates shuffle per vector from a splitmix64 stream seeded by `seed`
 * (test inputs; the reference's own generator, encrypt.c:40-85, draws m-bit
 * indices without rejecting those >= n). */
void o_random_errors(const o_params *p, uint64_t seed, size_t count, uint8_t *errs)
{
    const int n = p->n, t = p->t, nbytes = n / 8;
    uint16_t *perm = (uint16_t *)malloc((size_t)n * sizeof(uint16_t));
    if (!perm)
        return;
    uint64_t st = seed;
    for (size_t c = 0; c < count; c++) {
        uint8_t *e = errs + c * (size_t)nbytes;
        memset(e, 0, (size_t)nbytes);
        for (int i = 0; i < n; i++)
            perm[i] = (uint16_t)i;
        for (int i = 0; i < t; i++) {
            const int j = i + (int)(o_splitmix(&st) % (uint64_t)(n - i));
            const uint16_t x = perm[i];
            perm[i] = perm[j];
            perm[j] = x;
            e[perm[i] >> 3] |= (uint8_t)(1u << (perm[i] & 7));
        }
    }
    free(perm);
}
