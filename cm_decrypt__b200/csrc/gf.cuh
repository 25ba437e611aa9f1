// GF(2^m) arithmetic for the decrypt kernels, m = 12 (x^12+x^3+1) or
// m = 13 (x^13+x^4+x^3+x+1) -- the fields of CPU/param/param348864/src/gf.c
// and CPU/src/common/gf_13.c.
//
// Everything here is constant-time integer/XOR work: no tables, no branches
// on field values.  Two forms:
//   * scalar: one element in the low m bits of a u32 (plain per-stage path,
//     key expansion);
//   * bitsliced: an element spread over m u32 "planes", bit p of plane k being
//     bit k of the element held by lane-bit p -- 32 independent elements per
//     word, multiplied with AND-XOR networks (LOP3) across the planes.
#pragma once
#include <cstdint>

namespace cmd {

// ---------------------------------------------------------------- scalar --

// Folds a carry-less product of two field elements back below x^M.  Each
// fold replaces x^M by the low terms of the modulus; two folds suffice for
// products of degree <= 2M-2.
template <int M> __device__ __forceinline__ uint32_t gf_reduce(uint32_t p)
{
    if constexpr (M == 13) {
        uint32_t h = p >> 13;
        p = (p & 0x1FFFu) ^ h ^ (h << 1) ^ (h << 3) ^ (h << 4);
        h = p >> 13;
        p = (p & 0x1FFFu) ^ h ^ (h << 1) ^ (h << 3) ^ (h << 4);
    } else {
        uint32_t h = p >> 12;
        p = (p & 0xFFFu) ^ h ^ (h << 3);
        h = p >> 12;
        p = (p & 0xFFFu) ^ h ^ (h << 3);
    }
    return p;
}

// Shift-and-add product with the multiplier bits turned into all-ones /
// all-zero masks, so the instruction stream does not depend on the operands.
template <int M> __device__ __forceinline__ uint32_t gf_mul(uint32_t a, uint32_t b)
{
    uint32_t p = 0;
#pragma unroll
    for (int i = 0; i < M; i++)
        p ^= (a << i) & (0u - ((b >> i) & 1u));
    return gf_reduce<M>(p);
}

// The same product by integer multiplies on operands with holes (the
// constant-time "ctmul" construction of T. Pornin's BearSSL GHASH): a and b
// are split into four classes of bits, positions i = c (mod 4).  The integer
// product of two classes counts, at each position, the bit pairs that meet
// there; the four products landing on class k (i + j = k mod 4) sum to at
// most 13 pairs per position, below 16, so no count reaches the class's next
// position, and bit 0 of each count is the XOR.  16 multiply-adds (the FMA
// pipe) and about 25 logic operations instead of 13 shift-and-mask steps on
// the ALU pipe; multiplies take the same time for every operand.
template <int M> __device__ __forceinline__ uint32_t gf_mul_im(uint32_t a, uint32_t b)
{
    constexpr uint32_t K0 = 0x11111111u, K1 = K0 << 1, K2 = K0 << 2, K3 = K0 << 3;
    const uint32_t a0 = a & K0, a1 = a & K1, a2 = a & K2, a3 = a & K3;
    const uint32_t b0 = b & K0, b1 = b & K1, b2 = b & K2, b3 = b & K3;
    const uint32_t c0 = a0 * b0 + a1 * b3 + a2 * b2 + a3 * b1;
    const uint32_t c1 = a0 * b1 + a1 * b0 + a2 * b3 + a3 * b2;
    const uint32_t c2 = a0 * b2 + a1 * b1 + a2 * b0 + a3 * b3;
    const uint32_t c3 = a0 * b3 + a1 * b2 + a2 * b1 + a3 * b0;
    return gf_reduce<M>((c0 & K0) | (c1 & K1) | (c2 & K2) | (c3 & K3));
}

// Squaring is linear over GF(2): spread bit i to bit 2i, then reduce.
template <int M> __device__ __forceinline__ uint32_t gf_sq(uint32_t a)
{
    uint32_t x = a;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return gf_reduce<M>(x);
}

template <int M, int K> __device__ __forceinline__ uint32_t gf_sqn(uint32_t a)
{
#pragma unroll
    for (int i = 0; i < K; i++)
        a = gf_sq<M>(a);
    return a;
}

// a^(2^M - 2) (= 1/a, and 0 -> 0) with an Itoh-Tsujii style chain:
//   M = 13: a^3, a^15, a^255, a^4095, then one squaring  (4 mul, 12 sq)
//   M = 12: a^3, a^7, a^15, a^255, a^2047, then one squaring (5 mul, 12 sq)
// IM: the multiplies are gf_mul_im.
template <int M, bool IM = false> __device__ __forceinline__ uint32_t gf_inv(uint32_t a)
{
    auto mul = [](uint32_t x, uint32_t y) { return IM ? gf_mul_im<M>(x, y) : gf_mul<M>(x, y); };
    uint32_t a3 = mul(gf_sq<M>(a), a);
    if constexpr (M == 13) {
        uint32_t a15 = mul(gf_sqn<M, 2>(a3), a3);
        uint32_t a255 = mul(gf_sqn<M, 4>(a15), a15);
        uint32_t a4095 = mul(gf_sqn<M, 4>(a255), a15);
        return gf_sq<M>(a4095);
    } else {
        uint32_t a7 = mul(gf_sq<M>(a3), a);
        uint32_t a15 = mul(gf_sqn<M, 2>(a3), a3);
        uint32_t a255 = mul(gf_sqn<M, 4>(a15), a15);
        uint32_t a2047 = mul(gf_sqn<M, 3>(a255), a7);
        return gf_sq<M>(a2047);
    }
}

// num / den, the reference's gf_frac(den, num).
template <int M> __device__ __forceinline__ uint32_t gf_frac(uint32_t den, uint32_t num)
{
    return gf_mul<M>(gf_inv<M>(den), num);
}

// ------------------------------------------------------------- bitsliced --

// Reduction of a 2M-1 plane product in place (planes >= M folded down).
template <int M> __device__ __forceinline__ void bs_reduce(uint32_t *p)
{
    if constexpr (M == 13) {
#pragma unroll
        for (int k = 24; k >= 13; k--) {
            p[k - 9] ^= p[k];
            p[k - 10] ^= p[k];
            p[k - 12] ^= p[k];
            p[k - 13] ^= p[k];
        }
    } else {
#pragma unroll
        for (int k = 22; k >= 12; k--) {
            p[k - 9] ^= p[k];
            p[k - 12] ^= p[k];
        }
    }
}

// Unreduced schoolbook product accumulated into p[0..2M-2] (p ^= x*y).
template <int M> __device__ __forceinline__ void bs_mul_acc(uint32_t *p, const uint32_t *x, const uint32_t *y)
{
#pragma unroll
    for (int i = 0; i < M; i++)
#pragma unroll
        for (int j = 0; j < M; j++)
            p[i + j] ^= x[i] & y[j];
}

// o = x * y (o may alias x or y).
template <int M> __device__ __forceinline__ void bs_mul(uint32_t *o, const uint32_t *x, const uint32_t *y)
{
    uint32_t p[2 * M - 1];
#pragma unroll
    for (int k = 0; k < 2 * M - 1; k++)
        p[k] = 0;
    bs_mul_acc<M>(p, x, y);
    bs_reduce<M>(p);
#pragma unroll
    for (int k = 0; k < M; k++)
        o[k] = p[k];
}

// o = x^2: plane i moves to plane 2i, then the reduction.
template <int M> __device__ __forceinline__ void bs_sq(uint32_t *o, const uint32_t *x)
{
    uint32_t p[2 * M - 1];
#pragma unroll
    for (int k = 0; k < 2 * M - 1; k++)
        p[k] = (k & 1) ? 0u : x[k >> 1];
    bs_reduce<M>(p);
#pragma unroll
    for (int k = 0; k < M; k++)
        o[k] = p[k];
}

// o = x^(2^M-2) elementwise (0 -> 0), same chain as gf_inv.
template <int M> __device__ __forceinline__ void bs_inv(uint32_t *o, const uint32_t *x)
{
    uint32_t a3[M], t[M], a15[M];
    bs_sq<M>(t, x);
    bs_mul<M>(a3, t, x);
    if constexpr (M == 13) {
        bs_sq<M>(t, a3);
        bs_sq<M>(t, t);
        bs_mul<M>(a15, t, a3);
        bs_sq<M>(t, a15);
#pragma unroll
        for (int i = 0; i < 3; i++)
            bs_sq<M>(t, t);
        bs_mul<M>(t, t, a15);  // a^255
#pragma unroll
        for (int i = 0; i < 4; i++)
            bs_sq<M>(t, t);
        bs_mul<M>(t, t, a15);  // a^4095
        bs_sq<M>(o, t);
    } else {
        uint32_t a7[M];
        bs_sq<M>(t, a3);
        bs_mul<M>(a7, t, x);
        bs_sq<M>(t, a3);
        bs_sq<M>(t, t);
        bs_mul<M>(a15, t, a3);
        bs_sq<M>(t, a15);
#pragma unroll
        for (int i = 0; i < 3; i++)
            bs_sq<M>(t, t);
        bs_mul<M>(t, t, a15);  // a^255
#pragma unroll
        for (int i = 0; i < 3; i++)
            bs_sq<M>(t, t);
        bs_mul<M>(t, t, a7);   // a^2047
        bs_sq<M>(o, t);
    }
}

}  // namespace cmd
