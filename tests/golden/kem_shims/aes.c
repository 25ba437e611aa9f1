/* OpenSSL-backed AES-256 single-block ECB for the KEM fixture generator
 * (stands in for third_party/tiny-AES-c/aes.c).  Test-fixture tooling only. */
#include "aes.h"

#include <stdlib.h>
#include <string.h>
#include <openssl/evp.h>

void AES_init_ctx(struct AES_ctx *ctx, const uint8_t *key)
{
    memcpy(ctx->key, key, 32);
}

void AES_ECB_encrypt(const struct AES_ctx *ctx, uint8_t *buf)
{
    EVP_CIPHER_CTX *c = EVP_CIPHER_CTX_new();
    unsigned char out[32];
    int len = 0;
    if (!c || EVP_EncryptInit_ex(c, EVP_aes_256_ecb(), NULL, ctx->key, NULL) != 1)
        abort();
    EVP_CIPHER_CTX_set_padding(c, 0);
    if (EVP_EncryptUpdate(c, out, &len, buf, 16) != 1 || len != 16)
        abort();
    memcpy(buf, out, 16);
    EVP_CIPHER_CTX_free(c);
}
