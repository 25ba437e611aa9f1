/*
 * ref_keygen_harness.c -- thin C driver around the reference's own key
 * generation sources (somesh-vas/CM_Decrypt_ kem/common/core/sk_gen.c,
 * pk_gen.c, controlbits.c, root.c and kem/variant_<set>/gf.c, util.c),
 * compiled once per parameter set by oracle/Makefile into
 * oracle/_ref/libkeygen_<set>.so.  TEST INFRASTRUCTURE ONLY.
 *
 * crypto_kem_keypair (kem/common/core/operations.c:36-107) draws its seed from
 * randombytes and expands it with SHAKE256 from a third-party tree that the
 * reference does not ship; the tests do that expansion with Python's hashlib
 * and call the three stages below, which run the reference code unchanged.
 */
#include <stdint.h>

#include "controlbits.h"
#include "params.h"
#include "pk_gen.h"
#include "sk_gen.h"

#define API __attribute__((visibility("default")))

API int ref_kg_info(int *out6)
{
    out6[0] = GFBITS;
    out6[1] = SYS_N;
    out6[2] = SYS_T;
    out6[3] = PK_NROWS;
    out6[4] = PK_ROW_BYTES;
    out6[5] = COND_BYTES;
    return 0;
}

/* sk_gen.c:24-85: minimal polynomial of f in GF((2^m)^t); -1 if degree < t. */
API int ref_kg_genpoly(const uint16_t *f, uint16_t *irr)
{
    gf fc[SYS_T];
    for (int i = 0; i < SYS_T; i++)
        fc[i] = f[i];
    return genpoly_gen(irr, fc);
}

/* pk_gen.c:29-149: public key from the Goppa polynomial (t little-endian
 * coefficients, as stored in sk) and 2^m random 32-bit words; pi receives the
 * support permutation.  -1 when the draw is rejected. */
API int ref_kg_pk_gen(uint8_t *pk, const uint8_t *irr_bytes, const uint32_t *perm, int16_t *pi)
{
    unsigned char irr[IRR_BYTES];
    uint32_t pm[1 << GFBITS];
    for (int i = 0; i < IRR_BYTES; i++)
        irr[i] = irr_bytes[i];
    for (int i = 0; i < (1 << GFBITS); i++)
        pm[i] = perm[i];
    return pk_gen(pk, irr, pm, pi);
}

/* controlbits.c:180-220: Benes control bits of pi (COND_BYTES bytes). */
API void ref_kg_controlbits(uint8_t *out, const int16_t *pi)
{
    controlbitsfrompermutation(out, pi, GFBITS, 1 << GFBITS);
}
