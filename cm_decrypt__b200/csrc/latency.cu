// Latency-oriented decrypt path for the serving loop: tiles of up to 32
// ciphertexts of one parameter set, each ciphertext with its own key, in three
// launches per batch (any mix of sets: one tile per 32 ciphertexts of a set).
//
//  k_tile_tsynd  warp per ciphertext: the 2t syndromes (util.c:102-114) by the
//                transposed additive FFT, with no per-key syndrome table;
//  k_tile_bm     CTA per tile: the syndromes' last stage, Berlekamp-Massey
//                (bm.c:12-68) bitsliced across the tile, the locators' radix
//                conversion;
//  k_root_tile   warp per ciphertext: additive-FFT root search and the key's
//                support network (root_13.c:216-240).
//
// Syndromes.  synd() sums, over the ciphertext bits b < sb that are set, the
// table row L_b^j / g(L_b)^2 (j < 2t).  Written over the field: s_j =
// sum_a u_a a^j, with u_a = 1/g(a)^2 at the element a = L_b of every set bit
// and 0 elsewhere.  That is the transpose of evaluating a polynomial of 2^D'
// coefficients (2^D' >= 2t) at all 2^m elements, which the root search does
// with the additive FFT; so the syndromes come from the FFT run backwards:
//   1. the ciphertext bits, in support order, go through the key's support
//      network in reverse (the network maps FFT positions to support
//      positions; each layer is its own inverse), and select the key's
//      weights 1/g(a)^2 stored in FFT position order (KeyDev::wfft);
//   2. D' transposed butterfly levels, depth 0 first: A <- A + B,
//      B <- B + w*A (the transpose of A' = A + w*B, B' = A' + B);
//   3. each group of positions that shares its top D' bits is one word; the
//      word's parity per plane is the dual of the depth-D' constant of
//      sub-problem bitrev(word);
//   4. (in k_tile_bm, bitsliced across the tile) the transposed radix
//      conversion turns those 2^D' values into the power sums s_0 .. s_{2t-1}.
// All of it is exact GF(2^m) arithmetic, so the syndromes equal synd()'s.
// Per key it reads the support-network masks and the weights (about 39 KB
// for m = 13) instead of a 745 KB table, so the keys of a large serving set
// stay in L2.
//
// Scaled Berlekamp-Massey.  bm() updates C <- C + (d/b) x B, which needs
// b^-1 every iteration: a chain of ~16 dependent field operations per step.
// Here C <- b C + d x B instead, with the same decisions (d != 0, N >= 2L),
// the same truncation to t+1 coefficients and the same B/b/L updates.  By
// induction C_here = lambda * C_ref with lambda a product of earlier
// (nonzero) b values, so the returned polynomial is a nonzero multiple of
// bm()'s output: it has exactly the same roots and the decrypt flags exactly
// the same positions, decode failures included.  (The per-stage hook
// cmd_stage_bm keeps bm()'s exact output.)  Coefficients above the largest
// L of the tile are zero (deg C <= L), so they are neither multiplied into
// the discrepancy nor updated.
#include <algorithm>

#include "fft_root.cuh"
#include "gf.cuh"
#include "internal.h"

namespace cmd {

namespace {
constexpr uint32_t FULL = 0xFFFFFFFFu;
}

static_assert(sizeof(LatItem) == 40, "LatItem layout");

template <int S> struct TsDims {
    using F = FftDims<S>;
    static constexpr int M = F::M, T = F::T, NWD = F::NWD, R = F::R;
    static constexpr int DS = synd_depth(T);  // transposed-FFT depth, 2^DS >= 2t
    static constexpr int NS = 1 << DS;        // group sums per ciphertext
    static_assert(DS == M - 5, "the last transposed level pairs adjacent words: one group per word");
    static_assert(NS * 32 / 2 <= TILE_SUM_WORDS, "tile sums");
};

constexpr int TS_WARPS = 8;                  // ciphertexts per k_tile_tsynd CTA
constexpr size_t TS_FA_WORDS = 13 * 256;     // per-warp 2^m-element array, largest set

// One warp: the transposed FFT of ciphertext q of its tile; writes the
// group sums sums[s * 32 + q] (bit k = plane k), s < 2^D'.
template <int S>
__device__ __forceinline__ void tsynd_one(const LatItem &it, const uint8_t *__restrict__ cts,
                                          const uint32_t *__restrict__ tw, uint32_t *fa, uint16_t *sums, int q,
                                          int lane)
{
    using Z = TsDims<S>;
    using P = Set<S>;
    constexpr int M = Z::M, NWD = Z::NWD, R = Z::R, DS = Z::DS, SB = P::SB, CTW = P::CTW;
    static_assert(Z::NWD * M <= (int)TS_FA_WORDS, "transposed-FFT array");
    // 1. ciphertext bits in support order (word w = lane + 32j: positions
    //    32w .. 32w+31; bits >= sb are zero), then the network in reverse
    // (byte loads: a ciphertext may start at any byte; sb = 8 * ct bytes)
    static_assert(SB == 8 * P::CT, "synd() reads exactly the ciphertext's bytes");
    const uint8_t *c = cts + it.ct_off;
    uint32_t z[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
        const int w = lane + 32 * j;
        uint32_t v = 0;
        if (w < CTW) {
#pragma unroll
            for (int b = 0; b < 4; b++)
                if (4 * w + b < P::CT)
                    v |= (uint32_t)__ldg(c + 4 * w + b) << (8 * b);
        }
        z[j] = v;
    }
#pragma unroll
    for (int l = 2 * M - 2; l >= 0; l--)
        swap_layer<S>(z, it.bctl, l, lane);
    // 2a. depth 0 on u = bit * 1/g(a)^2: the pair (w, w + 2^(m-6)) is this
    //     lane's (z[j], z[j + R/2])
    const uint32_t *wf = it.wfft;
#pragma unroll
    for (int j = 0; j < R / 2; j++) {
        const int wa = lane + 32 * j, wb = wa + NWD / 2;
        const uint32_t *g = tw + (size_t)wa * 16;
        uint32_t A[M], B[M], G[M], p[2 * M - 1];
#pragma unroll
        for (int k = 0; k < M; k++) {
            B[k] = z[j + R / 2] & __ldg(wf + k * NWD + wb);
            A[k] = (z[j] & __ldg(wf + k * NWD + wa)) ^ B[k];
            G[k] = __ldg(g + k);
        }
#pragma unroll
        for (int k = 0; k < 2 * M - 1; k++)
            p[k] = 0;
        bs_mul_acc<M>(p, G, A);
        bs_reduce<M>(p);
        const int pa = fa_word(wa), pb = fa_word(wb);
#pragma unroll
        for (int k = 0; k < M; k++) {
            fa[k * NWD + pa] = A[k];
            fa[k * NWD + pb] = B[k] ^ p[k];
        }
    }
    __syncwarp();
    // 2b. depths 1 .. D'-2: pairs (wa, wa + Sw), Sw = 2^(m-d-6) words
#pragma unroll 1
    for (int d = 1; d < DS - 1; d++) {
        const int sbit = M - d - 6, Sw = 1 << sbit;
        const uint32_t *twd = tw + (size_t)(NWD - (NWD >> d)) * 16;
#pragma unroll 1
        for (int j = 0; j < R / 2; j++) {
            const int P2 = lane + 32 * j;
            const int wa = ((P2 >> sbit) << (sbit + 1)) | (P2 & (Sw - 1));
            const uint32_t *g = twd + (P2 & (Sw - 1)) * 16;
            const int pa = fa_word(wa), pb = fa_word(wa + Sw);
            uint32_t A[M], B[M], G[M], p[2 * M - 1];
#pragma unroll
            for (int k = 0; k < M; k++) {
                B[k] = fa[k * NWD + pb];
                A[k] = fa[k * NWD + pa] ^ B[k];
                G[k] = __ldg(g + k);
            }
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                p[k] = 0;
            bs_mul_acc<M>(p, G, A);
            bs_reduce<M>(p);
#pragma unroll
            for (int k = 0; k < M; k++) {
                fa[k * NWD + pa] = A[k];
                fa[k * NWD + pb] = B[k] ^ p[k];
            }
        }
        __syncwarp();
    }
    // 2c/3. depth D'-1 pairs adjacent words (one twiddle word); each word is
    //       a group: its parity per plane goes out as the sum of sub-problem
    //       bitrev_D'(word)
    {
        const uint32_t *g = tw + (size_t)(NWD - (NWD >> (DS - 1))) * 16;
        uint32_t G[M];
#pragma unroll
        for (int k = 0; k < M; k++)
            G[k] = __ldg(g + k);
#pragma unroll 1
        for (int j = 0; j < R / 2; j++) {
            const int wa = 2 * (lane + 32 * j);
            const int ia = fa_word(wa), ib = fa_word(wa + 1);
            uint32_t A[M], B[M], p[2 * M - 1];
#pragma unroll
            for (int k = 0; k < M; k++) {
                B[k] = fa[k * NWD + ib];
                A[k] = fa[k * NWD + ia] ^ B[k];
            }
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                p[k] = 0;
            bs_mul_acc<M>(p, G, A);
            bs_reduce<M>(p);
            uint32_t pa = 0, pb = 0;
#pragma unroll
            for (int k = 0; k < M; k++) {
                pa |= (uint32_t)(__popc(A[k]) & 1) << k;
                pb |= (uint32_t)(__popc(B[k] ^ p[k]) & 1) << k;
            }
            const int sa = (int)(__brev((uint32_t)wa) >> (32 - DS));
            const int sb = (int)(__brev((uint32_t)(wa + 1)) >> (32 - DS));
            sums[sa * 32 + q] = (uint16_t)pa;
            sums[sb * 32 + q] = (uint16_t)pb;
        }
    }
    __syncwarp();  // fa is refilled by this warp's next ciphertext, if any
}

// Four CTAs per tile; warp w of CTA c handles ciphertext 8c + w of the tile.
__global__ void __launch_bounds__(TS_WARPS * 32) k_tile_tsynd(const LatItem *__restrict__ items,
                                                              const uint8_t *__restrict__ cts,
                                                              uint32_t *__restrict__ scratch, FftPlans plans)
{
    extern __shared__ __align__(16) uint32_t smem_ts[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x >> 2, q = TS_WARPS * (blockIdx.x & 3) + warp, slot = 32 * t + q;
    const LatItem it = items[slot];
    if (it.set < 0 || q >= (int)items[(size_t)t * 32].pad)
        return;  // whole warp: no block-wide barrier follows
    uint16_t *sums = reinterpret_cast<uint16_t *>(scratch + (size_t)t * TILE_SCRATCH_WORDS + TILE_LOC_WORDS);
    uint32_t *fa = smem_ts + (size_t)warp * TS_FA_WORDS;
    switch (it.set) {
    case S348864: tsynd_one<S348864>(it, cts, plans.p[S348864].tw, fa, sums, q, lane); break;
    case S460896: tsynd_one<S460896>(it, cts, plans.p[S460896].tw, fa, sums, q, lane); break;
    case S6688128: tsynd_one<S6688128>(it, cts, plans.p[S6688128].tw, fa, sums, q, lane); break;
    case S6960119: tsynd_one<S6960119>(it, cts, plans.p[S6960119].tw, fa, sums, q, lane); break;
    default: tsynd_one<S8192128>(it, cts, plans.p[S8192128].tw, fa, sums, q, lane); break;
    }
}

// Threads of k_tile_bm: thread i owns locator coefficient i (t+1 <= 129).
constexpr int BM_WARPS = 5;
constexpr int BM_THREADS = BM_WARPS * 32;

template <int S> struct TileSmem {
    using Z = TsDims<S>;
    static constexpr int SS = Z::M | 1;  // odd plane stride: per-coefficient rows meet no bank conflicts
    uint32_t sx[Z::NS * SS];             // group sums -> syndromes -> converted locators
    uint32_t ring[(Z::T + 2) * SS];      // B, rotated one slot per step (the x*B shift)
    // Each warp's share of the discrepancy, plane k in word k (step parity):
    // plain stores, summed by every reader after the barrier.  (Shared
    // atomics from several warps onto the same 13 words serialise: about
    // 500 cycles a step on B200.)
    alignas(16) uint32_t wsum[2][BM_WARPS][16];
};

// The barrier of the warps that hold locator coefficients: the block
// barrier when all of them do, else named barrier 1 for the first NT threads.
template <int NT> __device__ __forceinline__ void bm_barrier()
{
    static_assert(NT % 32 == 0 && NT <= BM_THREADS, "whole warps");
    if constexpr (NT == BM_THREADS)
        __syncthreads();
    else
        asm volatile("bar.sync 1, %0;" ::"n"(NT) : "memory");
}

// Steps 1-2 of k_tile_bm, by the whole CTA: gather the tile's group sums
// (sx[s][k] bit q = plane k of sum s of ciphertext q; zero for q >= count),
// then the transposed radix conversion: sx[j] = syndrome j, bitsliced.
template <int S>
__device__ __forceinline__ void tile_syndromes(int count, const uint32_t *tile_scratch, TileSmem<S> &sm,
                                               const uint16_t *scalpow)
{
    using Z = TsDims<S>;
    constexpr int M = Z::M, NS = Z::NS, SS = TileSmem<S>::SS;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint16_t *sums = reinterpret_cast<const uint16_t *>(tile_scratch + TILE_LOC_WORDS);
    for (int s = warp; s < NS; s += BM_WARPS) {
        const uint32_t v = lane < count ? (uint32_t)sums[s * 32 + lane] : 0u;
        uint32_t mine = 0;
#pragma unroll
        for (int k = 0; k < M; k++) {
            const uint32_t b = __ballot_sync(FULL, (v >> k) & 1u);
            if (lane == k)
                mine = b;
        }
        if (lane < M)
            sm.sx[s * SS + lane] = mine;
    }
    __syncthreads();
    fft_convert_t<S, SS, BM_THREADS>(sm.sx, scalpow, tid, [] { __syncthreads(); });
}

template <int S>
__device__ __forceinline__ void tile_bm(int count, const uint32_t *tile_scratch, uint32_t *loc_bs,
                                        const uint16_t *scalpow, uint8_t *smem_raw)
{
    using Z = TsDims<S>;
    using Sm = TileSmem<S>;
    constexpr int M = Z::M, T = Z::T, NS = Z::NS, SS = Sm::SS, R = T + 2;
    static_assert(T + 1 <= BM_THREADS, "one thread per locator coefficient");
    Sm &sm = *reinterpret_cast<Sm *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // ---- 1-2. syndromes, bitsliced across the tile ------------------------
    for (int v = tid; v < R * SS; v += BM_THREADS)
        sm.ring[v] = (v == SS) ? FULL : 0u;  // B = x
    tile_syndromes<S>(count, tile_scratch, sm, scalpow);

    // ---- 3. scaled Berlekamp-Massey, thread i owns C_i -------------------
    // Warps 0 .. NWA-1 hold coefficients 0..t and run the loop on their own
    // named barrier (the fifth warp, needed only for t = 128, otherwise waits
    // at the block barrier after the loop).  Per step:
    //  (1) warps holding coefficients i <= max L form their shares
    //      C_i * S_{N-i}, XOR-reduce them across the warp (plane k to lane
    //      k) and store them; b * C_i, which needs no discrepancy, is formed
    //      in the same straight-line block, so it covers the reductions'
    //      latency;
    //  (2) barrier; every thread sums the warps' shares: d, bitsliced;
    //  (3) the owners of i <= hi form C_i <- b*C_i + d*B_i and B_i <- (N >=
    //      2L and d != 0) ? old C_i : B_i in the ring slot of coefficient i.
    //      hi = max(Lup, largest possible degree of B), with Lup = min(t,
    //      max(max L, N + 1 - min L)) a bound on every ciphertext's new L
    //      that is known before d is.  Coefficients above a ciphertext's new
    //      L come out zero (deg C <= L; b*C_i + d*B_i = 0 there), so a larger
    //      bound changes nothing, and above Lup the update is the swap alone.
    // The next step's decisions (mle = (d != 0) & (N >= 2L) from a mask of
    // the second condition, the new L, the tile's bounds) are lane bits and
    // warp reductions that overlap the update's multiplies.
    constexpr int NWA = (T + 32) / 32;  // warps holding coefficients 0..t
    static_assert(NWA <= BM_WARPS && 32 * NWA > T, "coefficient warps");
    const int i = tid;
    uint32_t C[M];
#pragma unroll
    for (int k = 0; k < M; k++)
        C[k] = (i == 0 && k == 0) ? FULL : 0u;
    __syncthreads();  // the syndromes and the ring are in place
    if (warp < NWA) {
        uint32_t bb[M];
#pragma unroll
        for (int k = 0; k < M; k++)
            bb[k] = k == 0 ? FULL : 0u;  // b = 1
        int Lq = 0, Bd = 1;              // lane q: L and a bound on deg B of ciphertext q
        int Lmax = 0, Lmin = 0, Bmax = 1;
        uint32_t geq = FULL;             // bit q: N >= 2 L_q
#pragma unroll 1
        for (int N = 0; N < 2 * T; N++) {
            // L <= N at step N, so lim = min(N, t, max L) is the tile's
            // largest L, and C_i = 0 for every i above it.
            const int lim = min(N, min(T, Lmax));
            const int Lup = min(T, max(Lmax, N + 1 - Lmin));
            uint32_t(*ws)[16] = sm.wsum[N & 1];
            uint32_t q1[2 * M - 1];  // b * C_i, unreduced (zero where C_i = 0)
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                q1[k] = 0;
            if (32 * warp <= lim) {
                // Lanes above lim multiply C_i = 0 (their row index is
                // clamped to stay inside the syndromes).
                uint32_t p[2 * M - 1], sv[M], v[M];
#pragma unroll
                for (int k = 0; k < 2 * M - 1; k++)
                    p[k] = 0;
                const uint32_t *src = sm.sx + max(N - i, 0) * SS;
#pragma unroll
                for (int k = 0; k < M; k++)
                    sv[k] = src[k];
                bs_mul_acc<M>(p, C, sv);
                bs_reduce<M>(p);
#pragma unroll
                for (int k = 0; k < M; k++)
                    v[k] = __reduce_xor_sync(FULL, p[k]);
                bs_mul_acc<M>(q1, bb, C);
                uint32_t mine = 0;
#pragma unroll
                for (int k = 0; k < M; k++)
                    mine = lane == k ? v[k] : mine;
                if (lane < M)
                    ws[warp][lane] = mine;
            }
            bm_barrier<NWA * 32>();
            // Ring entries this step touches: coefficients i <= hi (B_i, and
            // the swap), loaded before d so the loads overlap its sum.
            const int hi = max(Lup, min(Bmax, T));
            const bool own = i <= hi;
            int slot = i - N % R;
            slot = slot < 0 ? slot + R : slot;
            uint32_t *bp = sm.ring + slot * SS;
            uint32_t bv[M];
#pragma unroll
            for (int k = 0; k < M; k++)
                bv[k] = own ? bp[k] : 0u;
            // The buffer of step N is written again at step N + 2, after
            // every reader here has passed the next step's barrier.
            uint32_t d[M];
#pragma unroll
            for (int k = 0; k < M; k++)
                d[k] = 0;
#pragma unroll
            for (int w = 0; w < NWA; w++) {
                if (32 * w <= lim) {
                    const uint4 *src = reinterpret_cast<const uint4 *>(ws[w]);
#pragma unroll
                    for (int v = 0; v < (M + 3) / 4; v++) {
                        const uint4 x = src[v];
                        if (4 * v + 0 < M) d[4 * v + 0] ^= x.x;
                        if (4 * v + 1 < M) d[4 * v + 1] ^= x.y;
                        if (4 * v + 2 < M) d[4 * v + 2] ^= x.z;
                        if (4 * v + 3 < M) d[4 * v + 3] ^= x.w;
                    }
                }
            }
            uint32_t mne = 0;
#pragma unroll
            for (int k = 0; k < M; k++)
                mne |= d[k];
            const uint32_t mle = mne & geq;
            const bool my_mle = (mle >> lane) & 1u;
            const int Lnew = my_mle ? N + 1 - Lq : Lq;
            const int Bdnew = min(min(my_mle ? Lq : Bd, T) + 1, T);
            // the tile's bounds for the next step (lanes past `count` keep
            // L = 0 and never take the swap: their syndromes are zero)
            const int Lmax_n = (int)__reduce_max_sync(FULL, (unsigned)Lnew);
            const int Lmin_n = (int)__reduce_min_sync(FULL, lane < count ? (unsigned)Lnew : 0xFFFFu);
            const int Bmax_n = (int)__reduce_max_sync(FULL, lane < count ? (unsigned)Bdnew : 0u);
            const uint32_t geq_n = __ballot_sync(FULL, N + 1 >= 2 * Lnew);
            // C_i <- b*C_i + d*B_i for i <= hi; lanes above hi hold C_i = 0
            // and load B_i = 0, so they keep C_i = 0 and store nothing
            // (their slots belong to other coefficients).
            if (32 * warp <= hi) {
                bs_mul_acc<M>(q1, d, bv);
                bs_reduce<M>(q1);
#pragma unroll
                for (int k = 0; k < M; k++) {
                    if (own)
                        bp[k] = (bv[k] & ~mle) | (C[k] & mle);
                    C[k] = q1[k];
                }
            }
            // the slot that becomes coefficient 0 of x*B at step N+1
            const int freeslot = (R - (N + 1) % R) % R;
            if (tid < M)
                sm.ring[freeslot * SS + tid] = 0;
#pragma unroll
            for (int k = 0; k < M; k++)
                bb[k] = (bb[k] & ~mle) | (d[k] & mle);
            Lq = Lnew;
            Bd = Bdnew;
            Lmax = min(Lmax_n, T);
            Lmin = Lmin_n;
            Bmax = Bmax_n;
            geq = geq_n;
        }
    }
    __syncthreads();
    // ---- 4. radix conversion of the reversed locators, out ---------------
    // Entry x of the conversion array is C[T-x] (bm.c:62-65 reverses the
    // locator before root() evaluates it), zero for T < x < 2^D.
    using F = FftDims<S>;
    static_assert(F::NX <= NS && F::NX * 16 <= TILE_LOC_WORDS, "conversion array size");
    if (i <= T)
#pragma unroll
        for (int k = 0; k < M; k++)
            sm.sx[(T - i) * SS + k] = C[k];
    for (int v = tid; v < (F::NX - T - 1) * SS; v += BM_THREADS)
        sm.sx[(T + 1) * SS + v] = 0u;
    __syncthreads();
    fft_convert<S, SS, BM_THREADS>(sm.sx, scalpow, tid, [] { __syncthreads(); });
    for (int v = tid; v < F::NX * M; v += BM_THREADS) {
        const int x = v / M, k = v - x * M;
        loc_bs[x * 16 + k] = sm.sx[x * SS + k];
    }
}

__global__ void __launch_bounds__(BM_THREADS) k_tile_bm(const LatItem *__restrict__ items,
                                                        uint32_t *__restrict__ scratch, FftPlans plans)
{
    extern __shared__ __align__(16) uint8_t smem_tile[];
    const LatItem *ti = items + (size_t)blockIdx.x * 32;
    const int count = (int)ti[0].pad;
    uint32_t *tsc = scratch + (size_t)blockIdx.x * TILE_SCRATCH_WORDS;
    switch (ti[0].set) {
    case S348864: tile_bm<S348864>(count, tsc, tsc, plans.p[S348864].scalpow, smem_tile); break;
    case S460896: tile_bm<S460896>(count, tsc, tsc, plans.p[S460896].scalpow, smem_tile); break;
    case S6688128: tile_bm<S6688128>(count, tsc, tsc, plans.p[S6688128].scalpow, smem_tile); break;
    case S6960119: tile_bm<S6960119>(count, tsc, tsc, plans.p[S6960119].scalpow, smem_tile); break;
    default: tile_bm<S8192128>(count, tsc, tsc, plans.p[S8192128].scalpow, smem_tile); break;
    }
}

constexpr int ROOT_WARPS = 8;
constexpr size_t ROOT_FA_WORDS = 13 * 256;  // FftDims<S>::FA_WORDS, largest set

template <int S>
__device__ __forceinline__ void root_tile(const LatItem &it, const uint32_t *cv, int q, uint32_t *err,
                                          uint16_t *weight, const FftPlanDev &pl, uint32_t *fa)
{
    static_assert(FftDims<S>::FA_WORDS <= ROOT_FA_WORDS, "root array");
    const int lane = threadIdx.x & 31;
    // The row goes to the batch's error rows, or packed straight into the
    // request's own (host) buffer; the fence makes those stores visible to the
    // host before anything the stream writes after this kernel.
    const int cnt = fft_root_one<S, 16>(cv, q, fa, pl.tw, it.bctl, it.row ? nullptr : err + it.err_off, nullptr,
                                        lane, it.row);
    if (it.row)
        __threadfence_system();
    if (lane == 0 && weight)
        *weight = (uint16_t)cnt;
}

// Four CTAs per tile; warp w of CTA c handles ciphertext 8c + w of the tile.
__global__ void __launch_bounds__(ROOT_WARPS * 32) k_root_tile(const LatItem *__restrict__ items,
                                                               const uint32_t *__restrict__ loc_bs,
                                                               uint32_t *__restrict__ err,
                                                               uint16_t *__restrict__ weight, FftPlans plans)
{
    extern __shared__ __align__(16) uint32_t smem_root[];
    const int warp = threadIdx.x >> 5;
    const int t = blockIdx.x >> 2, q = ROOT_WARPS * (blockIdx.x & 3) + warp, slot = 32 * t + q;
    const LatItem it = items[slot];
    if (it.set < 0 || q >= (int)items[(size_t)t * 32].pad)
        return;  // whole warp: no block-wide barrier follows
    const uint32_t *cv = loc_bs + (size_t)t * TILE_SCRATCH_WORDS;
    uint32_t *fa = smem_root + (size_t)warp * ROOT_FA_WORDS;
    uint16_t *wp = weight ? weight + slot : nullptr;
    switch (it.set) {
    case S348864: root_tile<S348864>(it, cv, q, err, wp, plans.p[S348864], fa); break;
    case S460896: root_tile<S460896>(it, cv, q, err, wp, plans.p[S460896], fa); break;
    case S6688128: root_tile<S6688128>(it, cv, q, err, wp, plans.p[S6688128], fa); break;
    case S6960119: root_tile<S6960119>(it, cv, q, err, wp, plans.p[S6960119], fa); break;
    default: root_tile<S8192128>(it, cv, q, err, wp, plans.p[S8192128], fa); break;
    }
}

size_t tile_smem_bytes()
{
    size_t m = 0;
    m = std::max(m, sizeof(TileSmem<S348864>));
    m = std::max(m, sizeof(TileSmem<S460896>));
    m = std::max(m, sizeof(TileSmem<S6688128>));
    m = std::max(m, sizeof(TileSmem<S6960119>));
    m = std::max(m, sizeof(TileSmem<S8192128>));
    return m;
}

// Items of a single-key batch of `count` ciphertexts at a ct_bytes stride;
// error rows at an nw-word stride, row c = ciphertext c.
__global__ void k_tile_items(LatItem *__restrict__ items, uint32_t count, const uint32_t *wfft,
                             const uint32_t *bctl, uint32_t ct_bytes, uint32_t nw, int set, uint32_t nslots)
{
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslots)
        return;
    const uint32_t t = slot >> 5, q = slot & 31, left = count - 32 * t;
    const uint32_t cnt = left < 32 ? left : 32;
    items[slot] = LatItem{wfft, bctl, slot * ct_bytes, slot * nw, q < cnt ? set : -1, (int32_t)cnt, nullptr};
}

// The syndromes of every ciphertext of a tile as rows of 2t u16 (the
// per-stage hook's layout): steps 1-2 of k_tile_bm, then a transpose out.
template <int S>
__device__ __forceinline__ void synd_out(int count, const uint32_t *tsc, uint16_t *synd, const uint16_t *scalpow,
                                         uint8_t *smem_raw)
{
    using Sm = TileSmem<S>;
    constexpr int M = Set<S>::M, T = Set<S>::T;
    Sm &sm = *reinterpret_cast<Sm *>(smem_raw);
    tile_syndromes<S>(count, tsc, sm, scalpow);
    for (int v = threadIdx.x; v < count * 2 * T; v += BM_THREADS) {
        const int q = v / (2 * T), j = v - q * 2 * T;
        uint32_t x = 0;
#pragma unroll
        for (int k = 0; k < M; k++)
            x |= ((sm.sx[j * Sm::SS + k] >> q) & 1u) << k;
        synd[((size_t)blockIdx.x * 32 + q) * 2 * T + j] = (uint16_t)x;
    }
}

__global__ void __launch_bounds__(BM_THREADS) k_tile_synd_out(const LatItem *__restrict__ items,
                                                              const uint32_t *__restrict__ scratch,
                                                              uint16_t *__restrict__ synd, FftPlans plans)
{
    extern __shared__ __align__(16) uint8_t smem_tile[];
    const LatItem *ti = items + (size_t)blockIdx.x * 32;
    const int count = (int)ti[0].pad;
    const uint32_t *tsc = scratch + (size_t)blockIdx.x * TILE_SCRATCH_WORDS;
    switch (ti[0].set) {
    case S348864: synd_out<S348864>(count, tsc, synd, plans.p[S348864].scalpow, smem_tile); break;
    case S460896: synd_out<S460896>(count, tsc, synd, plans.p[S460896].scalpow, smem_tile); break;
    case S6688128: synd_out<S6688128>(count, tsc, synd, plans.p[S6688128].scalpow, smem_tile); break;
    case S6960119: synd_out<S6960119>(count, tsc, synd, plans.p[S6960119].scalpow, smem_tile); break;
    default: synd_out<S8192128>(count, tsc, synd, plans.p[S8192128].scalpow, smem_tile); break;
    }
}

cudaError_t tile_prepare(int dev, size_t smem, size_t ts_smem, size_t root_smem);

// The tile path over one key's batch (d_scratch: tile_single_scratch_words).
cudaError_t launch_tile_single(const KeyDev &k, const uint8_t *d_cts, size_t count, uint32_t *d_scratch,
                               uint32_t *d_err, uint16_t *d_weight, uint16_t *d_synd, const FftPlans &plans,
                               cudaStream_t s, LaunchCounter lc)
{
    if (count == 0)
        return cudaSuccess;
    const SetInfo si = set_info(k.set);
    const uint32_t ntiles = (uint32_t)((count + 31) / 32);
    LatItem *items = reinterpret_cast<LatItem *>(d_scratch);
    uint32_t *tiles = d_scratch + (size_t)ntiles * 32 * sizeof(LatItem) / 4;
    k_tile_items<<<(ntiles * 32 + 255) / 256, 256, 0, s>>>(items, (uint32_t)count, k.wfft, k.bctl, (uint32_t)si.ct,
                                                          (uint32_t)si.nw, k.set, ntiles * 32);
    lc.bump();
    if (d_synd) {
        int dev = 0;
        cudaGetDevice(&dev);
        const size_t smem = tile_smem_bytes();
        cudaError_t e = tile_prepare(dev, smem, TS_WARPS * TS_FA_WORDS * 4, ROOT_WARPS * ROOT_FA_WORDS * 4);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_synd_out, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return e;
        k_tile_tsynd<<<ntiles * (32 / TS_WARPS), TS_WARPS * 32, TS_WARPS * TS_FA_WORDS * 4, s>>>(items, d_cts, tiles,
                                                                                                plans);
        k_tile_synd_out<<<ntiles, BM_THREADS, smem, s>>>(items, tiles, d_synd, plans);
        lc.bump(2);
        return cudaGetLastError();
    }
    return launch_tile_path(items, d_cts, ntiles, tiles, d_err, d_weight, plans, s, lc);
}

size_t tile_single_scratch_words(size_t count)
{
    const size_t ntiles = (count + 31) / 32;
    return ntiles * 32 * sizeof(LatItem) / 4 + ntiles * TILE_SCRATCH_WORDS;
}

// Raises the tile kernels' shared-memory limits once per device.
cudaError_t tile_prepare(int dev, size_t smem, size_t ts_smem, size_t root_smem)
{
    static size_t attr[64] = {};
    size_t &set_to = attr[dev & 63];
    if (set_to >= smem)
        return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_tile_bm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tile_tsynd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ts_smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_root_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)root_smem);
    // One shared-memory split for all three kernels, so that CTAs of
    // concurrent batches' kernels can share an SM without it draining to
    // change its split.
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tile_tsynd, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_tile_bm, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_root_tile, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e == cudaSuccess)
        set_to = smem;
    return e;
}

// ntiles tiles of 32 item slots; weights are indexed by item slot.
cudaError_t launch_tile_path(const void *d_items, const uint8_t *d_cts, uint32_t ntiles, uint32_t *d_scratch,
                             uint32_t *d_err, uint16_t *d_weight, const FftPlans &plans, cudaStream_t s,
                             LaunchCounter lc)
{
    if (ntiles == 0)
        return cudaSuccess;
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = tile_smem_bytes();
    const size_t ts_smem = TS_WARPS * TS_FA_WORDS * 4;
    const size_t root_smem = ROOT_WARPS * ROOT_FA_WORDS * 4;
    if (cudaError_t e = tile_prepare(dev, smem, ts_smem, root_smem); e != cudaSuccess)
        return e;
    const LatItem *items = static_cast<const LatItem *>(d_items);
    k_tile_tsynd<<<ntiles * (32 / TS_WARPS), TS_WARPS * 32, ts_smem, s>>>(items, d_cts, d_scratch, plans);
    k_tile_bm<<<ntiles, BM_THREADS, smem, s>>>(items, d_scratch, plans);
    k_root_tile<<<ntiles * (32 / ROOT_WARPS), ROOT_WARPS * 32, root_smem, s>>>(items, d_scratch, d_err, d_weight,
                                                                             plans);
    lc.bump(3);
    return cudaGetLastError();
}

}  // namespace cmd
