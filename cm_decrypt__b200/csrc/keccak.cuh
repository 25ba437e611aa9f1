// Keccak-f[1600] for device code (FIPS 202): constants derived from their
// definitions at compile time, the permutation on 25 lanes held in
// registers.  Shared by SHAKE256 in decapsulation and key generation.
#pragma once
#include <cstdint>

namespace cmd {
namespace {

// ---- Keccak-f[1600] constants from their FIPS 202 definitions -----------
// rc(t): output bit of the LFSR x^8 + x^6 + x^5 + x^4 + 1 (FIPS 202 alg. 5).
constexpr bool rc_bit(int t)
{
    if (t % 255 == 0)
        return true;
    unsigned r = 1;  // R = 10000000 (bit 0 is the first position)
    for (int i = 1; i <= t % 255; i++) {
        unsigned r8 = r << 1;  // R = 0 || R
        const unsigned b8 = (r8 >> 8) & 1u;
        r8 ^= b8 | (b8 << 4) | (b8 << 5) | (b8 << 6);
        r = r8 & 0xFFu;
    }
    return r & 1u;
}
struct KeccakConst {
    uint64_t rc[24];
    int rot[25];  // offset of lane x + 5y
    constexpr KeccakConst() : rc(), rot()
    {
        for (int i = 0; i < 24; i++) {  // iota: RC[i], bit 2^j - 1 = rc(j + 7i)
            uint64_t v = 0;
            for (int j = 0; j <= 6; j++)
                if (rc_bit(j + 7 * i))
                    v |= 1ull << ((1 << j) - 1);
            rc[i] = v;
        }
        rot[0] = 0;  // rho: walk (x, y) = (1, 0) -> (y, 2x + 3y)
        int x = 1, y = 0;
        for (int t = 0; t < 24; t++) {
            rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
            const int nx = y, ny = (2 * x + 3 * y) % 5;
            x = nx;
            y = ny;
        }
    }
};
constexpr KeccakConst KC{};
static_assert(KC.rc[0] == 1 && KC.rot[1] == 1, "Keccak constants");
__constant__ uint64_t kRC[24] = {KC.rc[0],  KC.rc[1],  KC.rc[2],  KC.rc[3],  KC.rc[4],  KC.rc[5],
                                 KC.rc[6],  KC.rc[7],  KC.rc[8],  KC.rc[9],  KC.rc[10], KC.rc[11],
                                 KC.rc[12], KC.rc[13], KC.rc[14], KC.rc[15], KC.rc[16], KC.rc[17],
                                 KC.rc[18], KC.rc[19], KC.rc[20], KC.rc[21], KC.rc[22], KC.rc[23]};
// rho offset of lane (x, y), folded to a constant in the unrolled round.
__host__ __device__ constexpr int keccak_rot(int x0, int y0)
{
    if (x0 == 0 && y0 == 0)
        return 0;
    int x = 1, y = 0;
    for (int t = 0; t < 24; t++) {
        if (x == x0 && y == y0)
            return ((t + 1) * (t + 2) / 2) % 64;
        const int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    return 0;
}
static_assert(keccak_rot(1, 0) == KC.rot[1] && keccak_rot(4, 4) == KC.rot[24], "Keccak rotations");

__device__ __forceinline__ uint64_t rotl64(uint64_t v, int r) { return r ? (v << r) | (v >> (64 - r)) : v; }

__device__ __forceinline__ void keccak_f(uint64_t *A)
{
#pragma unroll 1
    for (int round = 0; round < 24; round++) {
        uint64_t C[5], B[25];
#pragma unroll
        for (int x = 0; x < 5; x++)
            C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) {
            const uint64_t D = C[(x + 4) % 5] ^ rotl64(C[(x + 1) % 5], 1);
#pragma unroll
            for (int y = 0; y < 5; y++)
                A[x + 5 * y] ^= D;
        }
        // rho and pi: B[y, 2x + 3y] = rotl(A[x, y], rot[x, y])
#pragma unroll
        for (int x = 0; x < 5; x++)
#pragma unroll
            for (int y = 0; y < 5; y++)
                B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(A[x + 5 * y], keccak_rot(x, y));
        // chi
#pragma unroll
        for (int y = 0; y < 5; y++)
#pragma unroll
            for (int x = 0; x < 5; x++)
                A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= kRC[round];
    }
}

}  // namespace
}  // namespace cmd
