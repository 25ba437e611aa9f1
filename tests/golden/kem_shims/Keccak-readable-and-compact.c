/* Stand-in for XKCP's CompactFIPS202 source that kem/common/core/
 * fips202_shim.c #includes (not shipped with the reference).  It defines the
 * one entry point that file uses, FIPS202_SHAKE256 (renamed by a macro there),
 * on top of OpenSSL's SHAKE256.  Test-fixture tooling only. */
#include <stdlib.h>
#include <openssl/evp.h>

void FIPS202_SHAKE256(const unsigned char *input, unsigned int inputByteLen,
                      unsigned char *output, int outputByteLen)
{
    EVP_MD_CTX *c = EVP_MD_CTX_new();
    if (!c || EVP_DigestInit_ex(c, EVP_shake256(), NULL) != 1 ||
        EVP_DigestUpdate(c, input, inputByteLen) != 1 ||
        EVP_DigestFinalXOF(c, output, (size_t)outputByteLen) != 1)
        abort();
    EVP_MD_CTX_free(c);
}
