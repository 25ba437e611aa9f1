#!/bin/sh
# Regenerates the reference's own KEM fixtures (kem/: one keypair per set from
# the fixed NIST-DRBG seed 0..47, then CT_PER_SK encapsulations) and the
# reference CPU decoder's errorstream for them.  Writes, per set:
#   tests/golden/kem/sk_<set>.bin, ct_<set>.bin, errorstream0_<set>.bin
#
# The two third-party pieces kem/ expects (tiny-AES-c, XKCP) are not shipped
# with the reference; kem_shims/ stands in for them with OpenSSL libcrypto.
# The regenerated sk_<set>.bin must equal the shipped one byte for byte (the
# known-answer check that pins the DRBG, SHAKE256, genpoly, pk_gen and
# controlbits path); the script fails otherwise.
#
# Usage: tests/golden/gen_kem_vectors.sh [CT_PER_SK] [REFERENCE_DIR]
# Needs the reference tree (read-only: the second argument, else
# $CMD_REFERENCE_DIR) and oracle/_ref/bin/decrypt_<set> (make -C oracle ref).
set -eu
CT_PER_SK="${1:-5}"
REF="${2:-${CMD_REFERENCE_DIR:-}}"
if [ -z "$REF" ] || [ ! -d "$REF/kem" ]; then
    echo "gen_kem_vectors.sh: give the reference tree as the second argument or in CMD_REFERENCE_DIR" >&2
    exit 2
fi
HERE="$(CDPATH= cd -- "$(dirname -- "$0")" && pwd)"
REPO="$(CDPATH= cd -- "$HERE/../.." && pwd)"
OUT="$HERE/kem"
SETS="348864 460896 6688128 6960119 8192128"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT

mkdir -p "$OUT"
cp -r "$REF/kem" "$TMP/kem"
chmod -R u+w "$TMP/kem"
mkdir -p "$TMP/third_party/tiny-AES-c" "$TMP/third_party/XKCP/Standalone/CompactFIPS202/C"
cp "$HERE/kem_shims/aes.h" "$HERE/kem_shims/aes.c" "$TMP/third_party/tiny-AES-c/"
cp "$HERE/kem_shims/Keccak-readable-and-compact.c" "$TMP/third_party/XKCP/Standalone/CompactFIPS202/C/"
rm -f "$TMP"/kem/test_vectors/Cipher_Sk/*.bin

for s in $SETS; do
    v="$TMP/kem/variant_$s"
    # Same compile line as kem/variant_<set>/build, plus -lcrypto for the shims
    # and without -march=native.
    (cd "$v" && gcc -O2 -w -I. -I../common/core -Isubroutines -DKAT \
        -DKATNUM="$(cat KATNUM)" -DCT_PER_SK="$CT_PER_SK" -DAES256=1 -DCBC=0 -DCTR=0 \
        "-DCRYPTO_NAMESPACE(x)=x" "-D_CRYPTO_NAMESPACE(x)=_##x" -o kat \
        ../common/kat_kem_vectors.c nist/rng.c ../common/core/controlbits.c \
        ../common/core/encrypt.c gf.c ../common/core/operations.c ../common/core/pk_gen.c \
        ../common/core/root.c ../common/core/sk_gen.c ../common/core/fips202_shim.c util.c \
        ../../third_party/tiny-AES-c/aes.c -ldl -lcrypto && ./kat)
    cmp "$TMP/kem/test_vectors/Cipher_Sk/sk_$s.bin" "$REF/kem/test_vectors/Cipher_Sk/sk_$s.bin"
    echo "sk_$s.bin: regenerated key equals the shipped key"
    cp "$TMP/kem/test_vectors/Cipher_Sk/sk_$s.bin" "$TMP/kem/test_vectors/Cipher_Sk/ct_$s.bin" "$OUT/"

    # Reference CPU decoder, unmodified, in the directory layout its fixed
    # relative paths expect (util.c: ../../../kem/test_vectors/Cipher_Sk,
    # decrypt.c: ../../results/output).
    run="$TMP/run_$s"
    mkdir -p "$run/CPU/param/param$s" "$run/CPU/results/output" "$run/kem/test_vectors"
    ln -s "$TMP/kem/test_vectors/Cipher_Sk" "$run/kem/test_vectors/Cipher_Sk"
    (cd "$run/CPU/param/param$s" && "$REPO/oracle/_ref/bin/decrypt_$s" "$CT_PER_SK" > /dev/null)
    cp "$run/CPU/results/output/errorstream0_$s.bin" "$OUT/errorstream0_$s.bin"
done
(cd "$OUT" && sha256sum *.bin > SHA256SUMS)
echo "fixtures written to $OUT"
