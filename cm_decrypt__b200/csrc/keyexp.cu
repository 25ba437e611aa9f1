// Secret-key expansion on the device: replaces the host-side initialisation()
// + support_gen() + compute_inverses() of the reference
// (CPU/param/param6960119/src/util.c:60-100, CPU/src/common/root_13.c:95-211).
//
// sk layout (util.c:60-72): [32 B seed][8 B pivots][t x LE u16 Goppa
// coefficients, low m bits][Benes control bits, (2m-1) * 2^(m-1) bits][s].
#include "gf.cuh"
#include "internal.h"

namespace cmd {

// m-bit reversal of i (the reference's bitrev: reverse 16 bits, drop 16-m).
template <int M> __device__ __forceinline__ uint32_t bitrev_m(uint32_t i)
{
    return __brev(i) >> (32 - M);
}

// Support generation.  The reference permutes the m bit-planes of the table
// bitrev(0..2^m-1) through a (2m-1)-layer Benes network (root_13.c:95-177).
// Element-wise the same network is: layer l exchanges entries p and p + 2^e
// (bit e of p clear; e = l for l < m, e = 2m-2-l after) when control bit
// l*2^(m-1) + q is set, q being p with bit e deleted.  One CTA holds all 2^m
// entries in shared memory; each thread owns 2^(m-1)/1024 exchanges per layer
// and performs them as masked XOR swaps (no branch on key bits).
template <int S> __global__ void __launch_bounds__(1024) k_support(KeyDev k)
{
    using P = Set<S>;
    constexpr int M = P::M;
    constexpr int SIZE = 1 << M, HALF = SIZE / 2;
    __shared__ uint16_t v[SIZE];
    const uint8_t *cond = k.sk + 40 + 2 * P::T;

    for (int p = threadIdx.x; p < SIZE; p += blockDim.x)
        v[p] = (uint16_t)bitrev_m<M>(p);
    for (int i = threadIdx.x; i <= P::T; i += blockDim.x)
        k.g[i] = (i == P::T) ? 1 : (uint16_t)((k.sk[40 + 2 * i] | (k.sk[41 + 2 * i] << 8)) & ((1 << M) - 1));
    __syncthreads();

    for (int layer = 0; layer < 2 * M - 1; layer++) {
        const int e = layer < M ? layer : 2 * M - 2 - layer;
        const uint32_t base = (uint32_t)layer * HALF;
        for (int q = threadIdx.x; q < HALF; q += blockDim.x) {
            const uint32_t p = ((q >> e) << (e + 1)) | (q & ((1u << e) - 1u));
            const uint32_t bit = base + q;
            const uint32_t c = 0u - ((cond[bit >> 3] >> (bit & 7)) & 1u);
            const uint32_t a = v[p], b = v[p + (1u << e)];
            const uint32_t d = (a ^ b) & c;
            v[p] = (uint16_t)(a ^ d);
            v[p + (1u << e)] = (uint16_t)(b ^ d);
        }
        __syncthreads();
    }
    for (int i = threadIdx.x; i < P::N; i += blockDim.x)
        k.L[i] = v[i];
}

// Per support point: g(L_i) by Horner (root_13.c:216-230), 1/g(L_i)^2, and for
// i < sb the syndrome-table row L_i^j / g(L_i)^2, j < 2t (util.c:86-100),
// packed two coefficients per 32-bit word (tab) and densely, m bits per
// coefficient (tabd).  Multiplies by integer multiplies on operands with holes
// (gf_mul_im).
template <int S> __global__ void __launch_bounds__(256) k_key_tables(KeyDev k)
{
    using P = Set<S>;
    constexpr int M = P::M, T = P::T;
    __shared__ uint16_t g[T + 1];
    for (int i = threadIdx.x; i <= T; i += blockDim.x)
        g[i] = k.g[i];
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P::N)
        return;
    const uint32_t a = k.L[i];
    uint32_t v = g[T];
    for (int j = T - 1; j >= 0; j--)
        v = gf_mul_im<M>(v, a) ^ g[j];
    const uint32_t inv = gf_inv<M, true>(gf_mul_im<M>(v, v));
    k.ginv2[i] = (uint16_t)inv;
    if (i < P::SB) {
        uint32_t x = inv;
        uint32_t *row = k.tab + (size_t)i * P::TWP;
        uint32_t *drow = k.tabd + (size_t)i * P::TWD;
        for (int w = P::TW; w < P::TWP; w++)
            row[w] = 0;
        // dense row: the 2t values' m bits back to back, little-endian
        uint64_t acc = 0;
        int nb = 0, dw = 0;
        for (int w = 0; w < P::TW; w++) {
            const uint32_t lo = x;
            x = gf_mul_im<M>(x, a);
            const uint32_t hi = x;
            x = gf_mul_im<M>(x, a);
            row[w] = lo | (hi << 16);
            acc |= (uint64_t)lo << nb;
            nb += M;
            acc |= (uint64_t)hi << nb;
            nb += M;
            while (nb >= 32) {
                drow[dw++] = (uint32_t)acc;
                acc >>= 32;
                nb -= 32;
            }
        }
        if (nb > 0)
            drow[dw++] = (uint32_t)acc;
        for (; dw < P::TWD; dw++)
            drow[dw] = 0;
    }
}

// Bitsliced support: warp w gathers the 32 points of word w and ballots each
// of the m bit-planes.  Points past n are zero (the kernels mask them off).
template <int S> __global__ void __launch_bounds__(256) k_bitslice_support(KeyDev k)
{
    using P = Set<S>;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= P::NW)
        return;
    const int i = 32 * w + lane;
    const uint32_t a = i < P::N ? k.L[i] : 0u;
#pragma unroll
    for (int b = 0; b < P::M; b++) {
        const uint32_t plane = __ballot_sync(0xFFFFFFFFu, (a >> b) & 1u);
        if (lane == 0)
            k.Lbs[b * P::NW + w] = plane;
    }
}

// The support network of k_support as per-word swap masks for the fused
// root search, which runs the same layers over a 2^m-bit array of zero flags
// (one bit per field element) instead of over 16-bit support entries.  Thread
// (layer, w) builds word w of layer l: bit b is control bit l*2^(m-1) + q of
// the pair whose lower element is p = 32w + b (bit e of p clear, q = p with
// bit e deleted), zero where bit e of p is set.
template <int S> __global__ void __launch_bounds__(256) k_benes_masks(KeyDev k)
{
    using P = Set<S>;
    constexpr int M = P::M, NWD = 1 << (M - 5), HALF = 1 << (M - 1);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (2 * M - 1) * NWD)
        return;
    const int layer = idx / NWD, w = idx % NWD;
    const int e = layer < M ? layer : 2 * M - 2 - layer;
    const uint8_t *cond = k.sk + 40 + 2 * P::T;
    uint32_t mask = 0;
    for (int b = 0; b < 32; b++) {
        const uint32_t p = 32u * w + b;
        const uint32_t q = ((p >> (e + 1)) << e) | (p & ((1u << e) - 1u));
        const uint32_t bit = (uint32_t)layer * HALF + q;
        const uint32_t c = (cond[bit >> 3] >> (bit & 7)) & 1u;
        mask |= (c & ~(p >> e)) << b;
    }
    k.bctl[idx] = mask;
}

// Syndrome weights in the additive FFT's position order, for the serving
// syndrome kernel (the transposed FFT): bit b of wfft[k * 2^(m-5) + w] = bit k
// of 1/g(a)^2 at the field element a = bitrev_m(32w + b), for all 2^m
// elements (the same values as compute_inverses' e_inv, util.c:86-100, there
// indexed by support position).  Thread per element, warp per word.
template <int S> __global__ void __launch_bounds__(256) k_fft_weights(KeyDev k)
{
    using P = Set<S>;
    constexpr int M = P::M, T = P::T, NWD = 1 << (M - 5);
    __shared__ uint16_t g[T + 1];
    for (int i = threadIdx.x; i <= T; i += blockDim.x)
        g[i] = k.g[i];
    __syncthreads();
    const uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;  // grid covers 2^m exactly
    const uint32_t a = __brev(y) >> (32 - M);
    uint32_t v = g[T];
    for (int j = T - 1; j >= 0; j--)
        v = gf_mul_im<M>(v, a) ^ g[j];
    const uint32_t inv = gf_inv<M, true>(gf_mul_im<M>(v, v));
    const int lane = threadIdx.x & 31, w = (int)(y >> 5);
#pragma unroll
    for (int b = 0; b < M; b++) {
        const uint32_t plane = __ballot_sync(0xFFFFFFFFu, (inv >> b) & 1u);
        if (lane == 0)
            k.wfft[b * NWD + w] = plane;
    }
}

cudaError_t launch_key_expand(const KeyDev &k, cudaStream_t s, LaunchCounter lc)
{
    return dispatch_set(k.set, [&]<int S>() -> cudaError_t {
        using P = Set<S>;
        k_support<S><<<1, 1024, 0, s>>>(k);
        k_key_tables<S><<<(P::N + 255) / 256, 256, 0, s>>>(k);
        k_bitslice_support<S><<<(P::NW * 32 + 255) / 256, 256, 0, s>>>(k);
        k_benes_masks<S><<<((2 * P::M - 1) * (1 << (P::M - 5)) + 255) / 256, 256, 0, s>>>(k);
        k_fft_weights<S><<<(1 << P::M) / 256, 256, 0, s>>>(k);
        lc.bump(5);
        return cudaGetLastError();
    });
}

}  // namespace cmd
