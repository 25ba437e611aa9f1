/* Stand-in for the tiny-AES-c header that kem/variant_<set>/nist/rng.c
 * includes (the submodule is not shipped with the reference).  Only the
 * single-block AES-256 ECB encryption the NIST DRBG uses is provided, backed
 * by OpenSSL libcrypto.  Test-fixture tooling only. */
#ifndef CMD_KEM_SHIM_AES_H
#define CMD_KEM_SHIM_AES_H
#include <stdint.h>

struct AES_ctx {
    uint8_t key[32];
};

void AES_init_ctx(struct AES_ctx *ctx, const uint8_t *key);
void AES_ECB_encrypt(const struct AES_ctx *ctx, uint8_t *buf);

#endif
