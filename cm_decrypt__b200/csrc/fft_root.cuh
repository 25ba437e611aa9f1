// Additive-FFT root search shared by the fused kernel and the serving tile
// path.  It replaces the reference's per-support-point Horner evaluation
// (CPU/src/common/root_13.c:216-240, eval at every L[i]) with an evaluation
// at all 2^m field elements followed by the key's support network, which is
// the permutation that generated L (root_13.c:95-177 applies it to the table
// bitrev(0..2^m-1)):
//
//  * fft_convert: radix conversion of up to 32 locators at once, bitsliced
//    across them (bit q of a word = locator q).  Entry x of the array holds
//    coefficient x of f(a) = sum_x C[T-x] a^x (the reversed locator the
//    reference evaluates).  Depth d: scale entry x by b_d^(x >> d), then
//    expand every stride-2^d sub-array in x^2 + x -- for block sizes n = 2^k
//    down to 4, third quarter ^= fourth, then second ^= third.  Afterwards
//    entry s holds the depth-D constant of the sub-problem whose Taylor
//    choices are the bits of s.
//  * fft_root_one: one warp, one locator q.  A 2^m-element bitsliced array
//    (plane-major, m planes of 2^(m-5) words, in shared memory) starts from
//    the depth-D constants -- position Y gets constant bitrev_D(Y >> (m-D)),
//    folded into the first butterfly level -- and takes D levels of
//    butterflies A' = A + w*B, B' = A' + B between whole words; position Y
//    then holds f(bitrev_m(Y)), which is where the support network expects
//    element Y's value (the last level feeds the zero test directly, without
//    storing the evaluations).  Zero flags (one bit per
//    element) go through the 2m-1 swap layers: pairs inside a word by
//    shifts, across lanes by shuffles, inside a lane by registers.  Bit j of
//    the result is "f(L[j]) == 0", the reference's error bit j.
//
// Tables: scalpow and the twiddle words come from fft_plan.cpp (per set),
// the swap masks from k_benes_masks (per key).
#pragma once
#include "gf.cuh"
#include "internal.h"

namespace cmd {

template <int S> struct FftDims {
    static constexpr int M = Set<S>::M, T = Set<S>::T, N = Set<S>::N, NW = Set<S>::NW;
    static constexpr int D = fft_depth(T);     // recursion depth, 2^D > T
    static constexpr int NX = 1 << D;          // radix-conversion entries
    static constexpr int NWD = 1 << (M - 5);   // words of a 2^m-bit array
    static constexpr int R = NWD / 32;         // of them per lane
    static constexpr int FA_WORDS = M * NWD;   // per-warp butterfly array
    static_assert(D <= M - 5, "butterflies must pair whole words");
};

// Where word w of a plane of the per-warp butterfly array is stored: odd
// 32-word rows keep their words with the bank bits inverted.  The butterfly
// levels that pair words less than 32 apart put lanes l and l + 16 in rows 2r
// and 2r + 1 at the same offsets; with the inversion those offsets fall in
// disjoint halves of the banks (offsets whose bit log2(distance) is 0 map to
// ones where it is 1), so no level meets a bank conflict.  Whole-row accesses
// stay a permutation of the banks.  Every read and write of the array goes
// through this map.
__device__ __forceinline__ int fa_word(int w) { return w ^ ((0 - ((w >> 5) & 1)) & 31); }

// Radix conversion of the bitsliced array cv[x * CVS + k] (x < 2^D, k < M),
// by NT cooperating threads (tid in [0, NT)); `sync` orders the steps.
template <int S, int CVS, int NT, class Sync>
__device__ __forceinline__ void fft_convert(uint32_t *cv, const uint16_t *__restrict__ scalpow, int tid, Sync sync)
{
    using F = FftDims<S>;
    constexpr int M = F::M, D = F::D, NX = F::NX;
#pragma unroll 1
    for (int d = 0; d < D; d++) {
        if (d > 0) {  // b_0 = 1: depth 0 needs no scaling
            for (int x = tid; x < NX; x += NT) {
                const uint32_t c = __ldg(scalpow + d * 256 + (x >> d));
                uint32_t v[M], cm[M], p[2 * M - 1];
#pragma unroll
                for (int k = 0; k < M; k++) {
                    v[k] = cv[x * CVS + k];
                    cm[k] = 0u - ((c >> k) & 1u);
                }
#pragma unroll
                for (int k = 0; k < 2 * M - 1; k++)
                    p[k] = 0;
                bs_mul_acc<M>(p, v, cm);
                bs_reduce<M>(p);
#pragma unroll
                for (int k = 0; k < M; k++)
                    cv[x * CVS + k] = p[k];
            }
            sync();
        }
#pragma unroll 1
        for (int kb = D - d; kb >= 2; kb--) {
            const int Q = 1 << (kb - 2);
#pragma unroll 1
            for (int h = 2; h >= 1; h--) {  // h = 2: third ^= fourth; h = 1: second ^= third
                for (int u = tid; u < (NX / 4) * M; u += NT) {
                    const int e = u / M, k = u - e * M;
                    const int sub = e & ((1 << d) - 1), rest = e >> d;
                    const int i = (rest >> (kb - 2)) * 4 * Q + h * Q + (rest & (Q - 1));
                    cv[((i << d) + sub) * CVS + k] ^= cv[(((i + Q) << d) + sub) * CVS + k];
                }
                sync();
            }
        }
    }
}

// Transpose of the radix conversion at depth D' = synd_depth(t) (2^D' >= 2t
// entries), for the serving path's syndromes: every elementary step of
// fft_convert (x_a ^= x_b, a scaling) is replaced by its transpose (x_b ^=
// x_a, the same scaling) and the steps run in the opposite order.  In:
// cv[s * CVS + k], the depth-D' constants' dual (sums over the FFT groups);
// out: entry x = the power sum of index x.
template <int S, int CVS, int NT, class Sync>
__device__ __forceinline__ void fft_convert_t(uint32_t *cv, const uint16_t *__restrict__ scalpow, int tid, Sync sync)
{
    constexpr int M = Set<S>::M, D = synd_depth(Set<S>::T), NX = 1 << D;
#pragma unroll 1
    for (int d = D - 1; d >= 0; d--) {
#pragma unroll 1
        for (int kb = 2; kb <= D - d; kb++) {
            const int Q = 1 << (kb - 2);
#pragma unroll 1
            for (int h = 1; h <= 2; h++) {  // h = 1: third ^= second; h = 2: fourth ^= third
                for (int u = tid; u < (NX / 4) * M; u += NT) {
                    const int e = u / M, k = u - e * M;
                    const int sub = e & ((1 << d) - 1), rest = e >> d;
                    const int i = (rest >> (kb - 2)) * 4 * Q + h * Q + (rest & (Q - 1));
                    cv[(((i + Q) << d) + sub) * CVS + k] ^= cv[((i << d) + sub) * CVS + k];
                }
                sync();
            }
        }
        if (d > 0) {
            for (int x = tid; x < NX; x += NT) {
                const uint32_t c = __ldg(scalpow + d * 256 + (x >> d));
                uint32_t v[M], cm[M], p[2 * M - 1];
#pragma unroll
                for (int k = 0; k < M; k++) {
                    v[k] = cv[x * CVS + k];
                    cm[k] = 0u - ((c >> k) & 1u);
                }
#pragma unroll
                for (int k = 0; k < 2 * M - 1; k++)
                    p[k] = 0;
                bs_mul_acc<M>(p, v, cm);
                bs_reduce<M>(p);
#pragma unroll
                for (int k = 0; k < M; k++)
                    cv[x * CVS + k] = p[k];
            }
            sync();
        }
    }
}

// Layer l of the key's support network over a 2^m-bit array held by one
// warp (word w = lane + 32j in z[j]): every pair (p, p + 2^e) whose mask bit
// (the lower element's) is set exchanges its two bits; e = l for l < m, else
// 2m-2-l.  A layer is its own inverse.
template <int S>
__device__ __forceinline__ void swap_layer(uint32_t *z, const uint32_t *__restrict__ bctl, int l, int lane)
{
    using F = FftDims<S>;
    constexpr int M = F::M, NWD = F::NWD, R = F::R;
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    const int e = l < M ? l : 2 * M - 2 - l;
    const uint32_t *ml = bctl + l * NWD;
    if (e < 5) {  // pairs inside a word
        const int sh = 1 << e;
#pragma unroll
        for (int j = 0; j < R; j++) {
            const uint32_t mk = __ldg(ml + lane + 32 * j);
            const uint32_t t = ((z[j] >> sh) ^ z[j]) & mk;
            z[j] ^= t ^ (t << sh);
        }
    } else if (e < 10) {  // pairs across lanes
        const int ls = 1 << (e - 5);
#pragma unroll
        for (int j = 0; j < R; j++) {
            const uint32_t other = __shfl_xor_sync(FULL, z[j], ls);
            const uint32_t mk = __ldg(ml + ((lane & ~ls) + 32 * j));
            z[j] ^= (z[j] ^ other) & mk;
        }
    } else {  // pairs inside a lane
        const int js = 1 << (e - 10);
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (!(j & js)) {
                const uint32_t mk = __ldg(ml + lane + 32 * j);
                const uint32_t t = (z[j] ^ z[j | js]) & mk;
                z[j] ^= t;
                z[j | js] ^= t;
            }
        }
    }
}

// Error row of n/8 bytes at byte address p (2-byte aligned), from the words
// v[j] = row word lane + 32j: 32-bit stores to 4-byte aligned addresses (a
// warp's store covers whole 128-byte lines), the row's odd 16-bit ends as
// 16-bit stores.  For a row that starts 2 bytes into a word, every stored
// word joins the upper half of row word k and the lower half of word k + 1
// (the next lane's, or lane 0's next word).  Used for host-mapped outputs,
// whose stores cross PCIe as they are made.
template <int S>
__device__ __forceinline__ void store_row_packed(uint8_t *p, const uint32_t *v, int lane)
{
    using F = FftDims<S>;
    constexpr int R = F::R, RB = F::N / 8;  // row bytes (even for every set)
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    static_assert(RB % 2 == 0, "rows of whole 16-bit units");
    if ((((uintptr_t)p) & 3) == 0) {
        uint32_t *o = reinterpret_cast<uint32_t *>(p);
#pragma unroll
        for (int j = 0; j < R; j++) {
            const int w = lane + 32 * j;
            if (w < RB / 4)
                o[w] = v[j];
            else if ((RB & 2) && w == RB / 4)
                *reinterpret_cast<uint16_t *>(p + 4 * w) = (uint16_t)v[j];
        }
    } else {
        if (lane == 0)
            *reinterpret_cast<uint16_t *>(p) = (uint16_t)v[0];
        uint32_t *o = reinterpret_cast<uint32_t *>(p + 2);
#pragma unroll
        for (int j = 0; j < R; j++) {
            const int k = lane + 32 * j;
            const uint32_t up = __shfl_down_sync(FULL, v[j], 1);
            const uint32_t wrap = __shfl_sync(FULL, j + 1 < R ? v[j + 1 < R ? j + 1 : j] : 0u, 0);
            const uint32_t nxt = lane == 31 ? wrap : up;
            if (k < (RB - 2) / 4)
                o[k] = (v[j] >> 16) | (nxt << 16);
            else if ((RB & 2) == 0 && k == (RB - 2) / 4)
                *reinterpret_cast<uint16_t *>(p + 2 + 4 * k) = (uint16_t)(v[j] >> 16);
        }
    }
}

// One warp: error row (and weight) of locator q from the converted array cv
// (bitsliced, cv[s * CVS + k]).  fa: this warp's FA_WORDS words of shared
// memory.  erow: NW words, or null.  epack: null, or the row's n/8 bytes
// packed (store_row_packed).  prow: null, or t+1 u16 that receive the
// weight, the flagged positions in ascending order and 0xFFFF in the unused
// slots (the weight never exceeds t: the reversed locator's leading
// coefficient is C[0], which the update never zeroes).  Returns the weight
// (all lanes).
template <int S, int CVS>
__device__ __forceinline__ int fft_root_one(const uint32_t *cv, int q, uint32_t *fa, const uint32_t *__restrict__ tw,
                                            const uint32_t *__restrict__ bctl, uint32_t *erow, uint16_t *prow,
                                            int lane, uint8_t *epack = nullptr)
{
    using F = FftDims<S>;
    constexpr int M = F::M, D = F::D, NWD = F::NWD, R = F::R, NW = F::NW;
    constexpr uint32_t FULL = 0xFFFFFFFFu;
    // Depth D-1: both operands are depth-D constants, read straight from cv.
    {
        constexpr int sbit = M - D - 5, Sw = 1 << sbit;
        const uint32_t *twd = tw + (size_t)((1 << (M - 5)) - (1 << (M - 5 - (D - 1)))) * 16;
#pragma unroll 1
        for (int j = 0; j < R / 2; j++) {
            const int P2 = lane + 32 * j;
            const int wa = ((P2 >> sbit) << (sbit + 1)) | (P2 & (Sw - 1));
            const int sa = (int)(__brev((uint32_t)(wa >> sbit)) >> (32 - D));
            const int sb = (int)(__brev((uint32_t)((wa + Sw) >> sbit)) >> (32 - D));
            const uint32_t *g = twd + (P2 & (Sw - 1)) * 16;
            uint32_t B[M], G[M], p[2 * M - 1];
#pragma unroll
            for (int k = 0; k < M; k++) {
                B[k] = 0u - ((cv[sb * CVS + k] >> q) & 1u);
                G[k] = __ldg(g + k);
            }
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                p[k] = 0;
            bs_mul_acc<M>(p, G, B);
            bs_reduce<M>(p);
            const int pa = fa_word(wa), pb = fa_word(wa + Sw);
#pragma unroll
            for (int k = 0; k < M; k++) {
                const uint32_t na = (0u - ((cv[sa * CVS + k] >> q) & 1u)) ^ p[k];
                fa[k * NWD + pa] = na;
                fa[k * NWD + pb] = na ^ B[k];
            }
        }
        __syncwarp();
    }
#pragma unroll
    for (int d = D - 2; d >= 1; d--) {
        const int sbit = M - d - 6, Sw = 1 << sbit;
        const uint32_t *twd = tw + (size_t)((1 << (M - 5)) - (1 << (M - 5 - d))) * 16;
#pragma unroll 1
        for (int j = 0; j < R / 2; j++) {
            const int P2 = lane + 32 * j;
            const int wa = ((P2 >> sbit) << (sbit + 1)) | (P2 & (Sw - 1));
            const uint32_t *g = twd + (P2 & (Sw - 1)) * 16;
            const int pa = fa_word(wa), pb = fa_word(wa + Sw);
            uint32_t A[M], B[M], G[M], p[2 * M - 1];
#pragma unroll
            for (int k = 0; k < M; k++) {
                A[k] = fa[k * NWD + pa];
                B[k] = fa[k * NWD + pb];
                G[k] = __ldg(g + k);
            }
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                p[k] = 0;
            bs_mul_acc<M>(p, G, B);
            bs_reduce<M>(p);
#pragma unroll
            for (int k = 0; k < M; k++) {
                const uint32_t na = A[k] ^ p[k];
                fa[k * NWD + pa] = na;
                fa[k * NWD + pb] = na ^ B[k];
            }
        }
        __syncwarp();
    }
    // Depth 0 pairs word w = lane + 32j with w + 2^(m-6): exactly the words
    // z[j] and z[j + R/2] of this lane, so the zero flags come straight from
    // the butterfly (no store of the evaluations).
    uint32_t z[R];
    {
        constexpr int Sw = 1 << (M - 6);
#pragma unroll
        for (int j = 0; j < R / 2; j++) {
            const int wa = lane + 32 * j;
            const uint32_t *g = tw + (size_t)wa * 16;  // depth 0: offset 0
            const int pa = fa_word(wa), pb = fa_word(wa + Sw);
            uint32_t A[M], B[M], G[M], p[2 * M - 1];
#pragma unroll
            for (int k = 0; k < M; k++) {
                A[k] = fa[k * NWD + pa];
                B[k] = fa[k * NWD + pb];
                G[k] = __ldg(g + k);
            }
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                p[k] = 0;
            bs_mul_acc<M>(p, G, B);
            bs_reduce<M>(p);
            uint32_t anya = 0, anyb = 0;
#pragma unroll
            for (int k = 0; k < M; k++) {
                const uint32_t na = A[k] ^ p[k];
                anya |= na;
                anyb |= na ^ B[k];
            }
            z[j] = ~anya;
            z[j + R / 2] = ~anyb;
        }
    }
    __syncwarp();  // fa may be refilled right after this call
#pragma unroll
    for (int l = 0; l < 2 * M - 1; l++)
        swap_layer<S>(z, bctl, l, lane);
    uint32_t v[R];
    int cnt = 0;
#pragma unroll
    for (int j = 0; j < R; j++) {
        const int w = lane + 32 * j;
        const int left = F::N - 32 * w;
        const uint32_t valid = left >= 32 ? FULL : (left > 0 ? ((1u << left) - 1u) : 0u);
        v[j] = z[j] & valid;
        if (erow && w < NW)
            erow[w] = v[j];
        cnt += __popc(v[j]);
    }
    if (epack)
        store_row_packed<S>(epack, v, lane);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        cnt += __shfl_xor_sync(FULL, cnt, off);
    if (prow) {
        // Word w = lane + 32j: its positions start after those of every word
        // with a smaller j, and of the lower lanes at the same j.  Every lane
        // walks all 32 bits of its words (predicated stores, no branch on the
        // error pattern).
        int base = 0;
#pragma unroll
        for (int j = 0; j < R; j++) {
            const int c = __popc(v[j]);
            int inc = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(FULL, inc, o);
                inc += lane >= o ? y : 0;
            }
            int off = base + inc - c;
            const int pos0 = 32 * (lane + 32 * j);
#pragma unroll 8
            for (int b = 0; b < 32; b++) {
                const int bit = (int)((v[j] >> b) & 1u);
                if (bit && off < F::T)
                    prow[1 + off] = (uint16_t)(pos0 + b);
                off += bit;
            }
            base += __shfl_sync(FULL, inc, 31);
        }
        for (int i = base + lane; i < F::T; i += 32)
            prow[1 + i] = 0xFFFFu;
        if (lane == 0)
            prow[0] = (uint16_t)cnt;
    }
    return cnt;
}

}  // namespace cmd
