// Fused, persistent decrypt kernel: syndrome -> Berlekamp-Massey -> root
// search -> error-word pack in one launch, for batches of one key or mixed
// batches of many keys and parameter sets.
//
// Work unit ("round"): up to WPB*32 ciphertexts of one key.  A CTA takes
// rounds from a device counter until none are left; each warp owns a tile of
// up to 32 of the round's ciphertexts (warp_share), so after the shared
// syndrome-table pipeline every warp runs independently:
//
//  1. stage its ciphertexts in shared memory (128-bit loads for a full
//     aligned tile of one slab, 16-bit loads for a partial one);
//  2. syndrome (util.c:102-114): lane q accumulates the 2t syndromes of
//     ciphertext q, m bits each back to back; the key's dense syndrome table
//     streams through shared memory four rows at a time (cp.async double
//     buffer, shared by all warps), the CTA forms the 16 XOR combinations of
//     each four rows, and each lane adds the combination its ciphertext's
//     four bits select (a read indexed by public ciphertext bits only);
//  3. transpose the syndromes to bitsliced form (bit q = ciphertext q) by a
//     shuffle butterfly;
//  4. Berlekamp-Massey (bm.c:12-68) bitsliced across the 32 ciphertexts: lane
//     l owns locator coefficients l, l+32, ... (kept in shared memory, so the
//     per-step loop over them stays rolled and small), the discrepancy is a
//     redux XOR reduction, B lives in a shared ring buffer whose rotation
//     implements the x*B shift.  The update is the scaled form C <- b*C +
//     d*x*B instead of bm()'s C <- C + (d/b)*x*B: same decisions (d != 0,
//     N >= 2L), same truncation, and by induction the result is lambda times
//     bm()'s locator with lambda a product of nonzero b values -- the same
//     roots, so the same flagged positions, with no inversion chain per step.
//     deg C <= L for every ciphertext, so only coefficients up to the tile's
//     largest L enter the discrepancy and the update (about half the slots
//     of the reference loop bounds for weight-t errors, where L ~ N/2);
//  5. root search (root_13.c:216-240 evaluates the locator at each support
//     point): the locator is evaluated at all 2^m field elements by an
//     additive FFT, then the key's support network (the Benes layers that
//     generate the support, root_13.c:95-177) carries the zero flags to
//     support order:
//     a. radix conversion (scalings g(x) = f(b_d x) and Taylor expansions in
//        x^2 + x, depth by depth), bitsliced across the 32 ciphertexts;
//     b. per ciphertext: a 2^m-element bitsliced array (m planes of 2^(m-5)
//        words) starts from the D-th-level constants and takes D levels of
//        butterflies A' = A + w*B, B' = A' + B between whole words;
//     c. zero flags -> the key's 2m-1 swap layers (word swaps across lanes
//        by shuffle, inside a lane by register, inside a word by shifts) ->
//        the packed error row and its weight.
//     The tables of the recursion are per set (fft_plan.cpp).
#pragma once
#include "fft_root.cuh"
#include "gf.cuh"
#include "internal.h"

namespace cmd {

constexpr uint32_t FULLMASK = 0xFFFFFFFFu;
constexpr int GROUP_ROWS = 4;  // syndrome-table rows combined per step (16 XOR combinations)

__host__ __device__ constexpr int cmax(int a, int b) { return a > b ? a : b; }
__host__ __device__ constexpr int al16(int x) { return (x + 15) / 16 * 16; }

template <int S> struct Fz {
    using P = Set<S>;
    static constexpr int M = P::M, T = P::T, NJ = (T + 1 + 31) / 32;
    static constexpr int TWD = P::TWD;               // dense table row (words)
    static constexpr int RING = T + 2;               // B ring slots
    static constexpr int NX = FftDims<S>::NX;        // radix-conversion entries
    static constexpr int RAW_B = 32 * P::CT;
    static constexpr int RING_B = RING * M * 4;
    static constexpr int FA_B = FftDims<S>::FA_WORDS * 4;  // root-search array
    static constexpr int CM_B = (T + 1) * M * 4;     // BM locator, after the ring
    static constexpr int A_B = al16(cmax(cmax(RAW_B + 16, RING_B + CM_B), FA_B));
    static constexpr int S_B = al16(2 * T * M * 4);  // bitsliced syndromes / locator
    static constexpr int WARP_B = A_B + S_B;
    static constexpr int NWU = (2 * T * M + 31) / 32;  // syndrome accumulator words in use
    static constexpr int CS = NWU | 1;  // combination row stride: odd, so the 16 rows lanes pick meet distinct banks
    // the CTA's syndrome region: two staged groups of table rows, then the
    // group's 16 XOR combinations
    static constexpr int SYN_B = al16((2 * GROUP_ROWS * TWD + 16 * CS) * 4);
    static_assert(P::SB % GROUP_ROWS == 0, "whole groups of ciphertext bits");
    static_assert(NX * M * 4 <= S_B, "conversion array must fit the syndrome region");
};

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    const uint32_t s = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Little-endian 32-bit read at any byte offset of shared memory.
__device__ __forceinline__ uint32_t ld_u32_any(const uint8_t *p)
{
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~(uintptr_t)3);
    const uint32_t sh = (uint32_t)(a & 3) * 8;
    return __funnelshift_r(w[0], w[1], sh);
}

struct RoundCtx {
    const FusedArgs *a;
    FusedTile tile;
    FusedKeyRef key;
};

// Which ciphertexts of a round warp `warp` takes: *first (offset in the
// round) and the count.  Rounds of more than 16*WPB ciphertexts are spread
// evenly over the WPB warps (each takes 32 or fewer); smaller ones are packed
// into whole 32-ciphertext tiles.  Per warp, Berlekamp-Massey costs the same
// for any fill while the root search costs per ciphertext, and the two warps
// that share a scheduler set a round's time: once packing would put two full
// tiles on one scheduler, an even spread shortens the round (a round of 224
// on 8 warps: 28 each instead of 32 on seven warps and none on one).
template <int WPB> __device__ __forceinline__ int warp_share(uint32_t count, int warp, uint32_t *first)
{
    if (count > 16u * WPB) {
        const uint32_t base = count / WPB, extra = count % WPB;
        *first = warp * base + min((uint32_t)warp, extra);
        return (int)(base + ((uint32_t)warp < extra ? 1u : 0u));
    }
    const int rem = (int)count - warp * 32;
    *first = (uint32_t)warp * 32;
    return rem < 0 ? 0 : (rem > 32 ? 32 : rem);
}

// Index (in the batch) of ciphertext q of the warp whose share starts at
// offset `first` of this round.
__device__ __forceinline__ uint64_t ct_index(const RoundCtx &rc, uint32_t first, int q)
{
    const uint64_t slot = rc.tile.first + first + q;
    return rc.a->order ? rc.a->order[slot] : slot;
}

template <int S, int WPB>
__device__ __forceinline__ void fused_round(const RoundCtx &rc, uint8_t *smem)
{
    using Z = Fz<S>;
    using P = Set<S>;
    constexpr int M = Z::M, T = Z::T, TWD = Z::TWD, NW = P::NW;
    const FusedArgs &a = *rc.a;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t wfirst;
    const int ntile = warp_share<WPB>(rc.tile.count, warp, &wfirst);

    uint32_t *tabbuf = reinterpret_cast<uint32_t *>(smem);
    uint8_t *wbase = smem + Z::SYN_B + warp * Z::WARP_B;
    uint8_t *raw = wbase;                                            // phase 1-2
    uint32_t *ring = reinterpret_cast<uint32_t *>(wbase);            // phase 4
    uint32_t *fa = reinterpret_cast<uint32_t *>(wbase);              // phase 5
    uint32_t *sS = reinterpret_cast<uint32_t *>(wbase + Z::A_B);     // phase 3-4
    uint32_t *cv = sS;                                               // phase 4-5
    const uint32_t *tab = rc.key.tab;

    // ---- 1. stage ciphertexts --------------------------------------------
    if (!a.order && !a.ct_off) {
        // one slab: 128-bit loads for a whole aligned tile, else 16-bit loads
        // (every set's ciphertext length is even)
        const uint8_t *src = a.cts + ct_index(rc, wfirst, 0) * P::CT;
        if (ntile == 32 && (((uintptr_t)src) & 15) == 0) {
            for (int v = lane; v < Z::RAW_B / 16; v += 32)
                reinterpret_cast<uint4 *>(raw)[v] = __ldg(reinterpret_cast<const uint4 *>(src) + v);
        } else {
            const uint16_t *s16 = reinterpret_cast<const uint16_t *>(src);
            for (int v = lane; v < ntile * P::CT / 2; v += 32)
                reinterpret_cast<uint16_t *>(raw)[v] = __ldg(s16 + v);
        }
    } else {
        for (int q = 0; q < ntile; q++) {
            const uint64_t c = ct_index(rc, wfirst, q);
            const uint8_t *src = a.cts + (a.ct_off ? a.ct_off[c] : c * (uint64_t)P::CT);
            for (int v = lane; v < P::CT; v += 32)
                raw[q * P::CT + v] = src[v];
        }
    }
    for (int v = ntile * P::CT + lane; v < Z::RAW_B; v += 32)
        raw[v] = 0;
    if (lane < 4)
        reinterpret_cast<uint32_t *>(raw + Z::RAW_B)[lane] = 0;  // tail read by ld_u32_any
    __syncwarp();

    // ---- 2. syndrome -----------------------------------------------------
    // The key's dense table: row b holds the 2t values L_b^j / g(L_b)^2 as m
    // bits each, back to back (bit j*m + k = bit k of value j), so lane q's
    // accumulator word w holds bits 32w .. 32w+31 of ciphertext q's 2t*m
    // syndrome bits.  The rows go in groups of four: the CTA forms the 16
    // XOR combinations of a group once (combination x = the rows whose bit is
    // set in x), and each lane adds the one its ciphertext's four bits select
    // -- one load and one XOR per word instead of four masked XORs.  Rows of
    // the next group are staged by cp.async meanwhile.
    constexpr int NWU = Z::NWU, CS = Z::CS, G = GROUP_ROWS;
    constexpr int NG = P::SB / G;
    uint32_t acc[NWU];
#pragma unroll
    for (int w = 0; w < NWU; w++)
        acc[w] = 0;
    uint32_t *comb = tabbuf + 2 * G * TWD;  // [16][CS]
    auto stage = [&](int g) {  // rows of group g into buffer g & 1: TWD 16-byte pieces
        if (tid < TWD)
            cp_async16(tabbuf + (g & 1) * G * TWD + 4 * tid, tab + (size_t)g * G * TWD + 4 * tid);
        cp_async_commit();
    };
    stage(0);
    const uint8_t *myct = raw + lane * P::CT;
    uint32_t ctw = 0;
#pragma unroll 1
    for (int g = 0; g < NG; g++) {
        cp_async_wait<0>();
        __syncthreads();  // group g's rows are in; every lane is done with group g-1's combinations
        if (g + 1 < NG)
            stage(g + 1);
        if (tid < NWU) {
            const uint32_t *rows = tabbuf + (g & 1) * G * TWD + tid;
            const uint32_t r0 = rows[0], r1 = rows[TWD], r2 = rows[2 * TWD], r3 = rows[3 * TWD];
            const uint32_t c3 = r0 ^ r1, c5 = r2 ^ r0, c6 = r2 ^ r1, c7 = r2 ^ c3;
            uint32_t *o = comb + tid;
            o[0 * CS] = 0u;
            o[1 * CS] = r0;
            o[2 * CS] = r1;
            o[3 * CS] = c3;
            o[4 * CS] = r2;
            o[5 * CS] = c5;
            o[6 * CS] = c6;
            o[7 * CS] = c7;
            o[8 * CS] = r3;
            o[9 * CS] = r3 ^ r0;
            o[10 * CS] = r3 ^ r1;
            o[11 * CS] = r3 ^ c3;
            o[12 * CS] = r3 ^ r2;
            o[13 * CS] = r3 ^ c5;
            o[14 * CS] = r3 ^ c6;
            o[15 * CS] = r3 ^ c7;
        }
        __syncthreads();  // the combinations are in
        const int b = g * G;  // a multiple of 4: the group's bits share one ciphertext word
        if ((b & 31) == 0)
            ctw = ld_u32_any(myct + (b >> 3));
        const uint32_t *pick = comb + ((ctw >> (b & 31)) & 15u) * CS;
#pragma unroll
        for (int w = 0; w < NWU; w++)
            acc[w] ^= pick[w];
    }
    if (ntile == 0)
        return;  // no work for this warp in this round (the CTA-wide part is done)

    // ---- 3. transpose: sS[j*M + k] bit q = bit k of syndrome j of ct q ----
    // Syndrome bit x = j*M + k is bit x mod 32 of accumulator word x / 32.
    // Each accumulator word is a 32x32 bit matrix (row q = lane q's word),
    // and sS wants its transpose: five butterfly steps, each swapping the
    // off-diagonal blocks of one size (16, 8, 4, 2, 1 columns) between lanes
    // l and l ^ j, leave bit b of every ciphertext in lane b.  (One shuffle
    // and four logic operations a step, against 32 ballots and selects.)
    {
        constexpr uint32_t M0[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
        uint32_t keep[5];  // per step: the columns this lane keeps
#pragma unroll
        for (int st = 0; st < 5; st++)
            keep[st] = (lane & (16 >> st)) ? ~M0[st] : M0[st];
#pragma unroll
        for (int w = 0; w < NWU; w++) {
            uint32_t v = acc[w];
#pragma unroll
            for (int st = 0; st < 5; st++) {
                const int j = 16 >> st;
                const uint32_t x = __shfl_xor_sync(FULLMASK, v, j);
                const uint32_t t = (lane & j) ? (x >> j) : (x << j);
                v = (v & keep[st]) | (t & ~keep[st]);
            }
            if (32 * w + lane < 2 * T * M)
                sS[32 * w + lane] = v;
        }
    }
    __syncwarp();

    // ---- 4. Berlekamp-Massey, bitsliced across the 32 ciphertexts --------
    {
        constexpr int NJ = Z::NJ, R = Z::RING;
        uint32_t *sCm = ring + R * M;  // locator coefficients [T+1][M]
        for (int v = lane; v < (T + 1) * M; v += 32)
            sCm[v] = (v == 0) ? FULLMASK : 0u;  // C = 1
        for (int v = lane; v < R * M; v += 32)
            ring[v] = (v == M) ? FULLMASK : 0u;  // B = x
        uint32_t bb[M];
#pragma unroll
        for (int k = 0; k < M; k++)
            bb[k] = k == 0 ? FULLMASK : 0u;       // b = 1
        int Lq = 0;                               // L of ciphertext `lane`
        int Bd = 1;                               // bound on deg B of ciphertext `lane`
        int Lmax = 0, Bmax = 1;                   // their maxima over the tile
        __syncwarp();
#pragma unroll 1
        for (int N = 0; N < 2 * T; N++) {
            // deg C <= L for every ciphertext, so coefficients above the
            // tile's largest L are zero: they take no part in the discrepancy
            const int lim = min(N, min(T, Lmax));
            uint32_t p[2 * M - 1];
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                p[k] = 0;
#pragma unroll 1
            for (int j = 0; 32 * j <= lim; j++) {
                const int i = lane + 32 * j;
                if (i <= lim) {
                    const uint32_t *sv = sS + (N - i) * M;
                    const uint32_t *cp = sCm + i * M;
                    uint32_t s[M], c[M];
#pragma unroll
                    for (int k = 0; k < M; k++) {
                        s[k] = sv[k];
                        c[k] = cp[k];
                    }
                    bs_mul_acc<M>(p, c, s);
                }
            }
            bs_reduce<M>(p);
            uint32_t d[M];
            uint32_t mne = 0;
#pragma unroll
            for (int k = 0; k < M; k++) {
                const uint32_t v = __reduce_xor_sync(FULLMASK, p[k]);
                d[k] = v;
                mne |= v;
            }
            const bool my_mle = ((mne >> lane) & 1u) && (N >= 2 * Lq);
            const uint32_t mle = __ballot_sync(FULLMASK, my_mle);
            const int Bdn = min(min(my_mle ? Lq : Bd, T) + 1, T);
            Lq = my_mle ? N + 1 - Lq : Lq;
            const int Lb = min((int)__reduce_max_sync(FULLMASK, (unsigned)Lq), T);
            const int Bm = min(Bmax, T);
            // Scaled update C <- b*C + d*x*B (see the note at the top of the
            // file): both products accumulate unreduced, one reduction.
            // After the step deg C <= L, so coefficients above the tile's
            // new largest L stay zero; B there only takes the swap (to C_i =
            // 0) where its degree bound reaches, and is zero above that.
            int off = (R - (N % R)) % R;  // slot(i) = (i - N) mod R
            const int hi = Lb > Bm ? Lb : Bm;
#pragma unroll 1
            for (int j = 0; j < NJ && 32 * j <= hi; j++) {
                const int i = lane + 32 * j;
                if (i > Lb && i <= Bm) {
                    int slot = i + off;
                    slot = slot >= R ? slot - R : slot;
                    uint32_t *bp = ring + slot * M;
#pragma unroll
                    for (int k = 0; k < M; k++)
                        bp[k] &= ~mle;
                } else if (i <= Lb) {
                    int slot = i + off;
                    slot = slot >= R ? slot - R : slot;
                    uint32_t *bp = ring + slot * M;
                    uint32_t *cp = sCm + i * M;
                    uint32_t bv[M], oc[M], q[2 * M - 1];
#pragma unroll
                    for (int k = 0; k < M; k++) {
                        bv[k] = bp[k];
                        oc[k] = cp[k];
                    }
#pragma unroll
                    for (int k = 0; k < 2 * M - 1; k++)
                        q[k] = 0;
                    bs_mul_acc<M>(q, bb, oc);
                    bs_mul_acc<M>(q, d, bv);
                    bs_reduce<M>(q);
#pragma unroll
                    for (int k = 0; k < M; k++) {
                        cp[k] = q[k];
                        bp[k] = (bv[k] & ~mle) | (oc[k] & mle);
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < M; k++)
                bb[k] = (bb[k] & ~mle) | (d[k] & mle);
            const int freeslot = (R - ((N + 1) % R)) % R;
            if (lane < M)
                ring[freeslot * M + lane] = 0;
            Bd = Bdn;
            Lmax = Lb;
            // (lanes past the tile's count never take the swap: zero syndromes)
            Bmax = (int)__reduce_max_sync(FULLMASK, lane < ntile ? (unsigned)Bd : 0u);
            __syncwarp();
        }
        // The reference's root search evaluates sum_x C[T-x] a^x
        // (bm.c:62-65 reverses the locator): entry x of the conversion array
        // is C[T-x], zero for T < x < 2^D.
        for (int v = lane; v < (T + 1) * M; v += 32) {
            const int i = v / M, k = v - i * M;
            cv[(T - i) * M + k] = sCm[v];
        }
        for (int v = lane; v < (Z::NX - T - 1) * M; v += 32)
            cv[(T + 1) * M + v] = 0u;
        __syncwarp();
    }

    // ---- 5. root search (fft_root.cuh) -------------------------------------
    const FftPlanDev pl = a.fft[S];
    fft_convert<S, M, 32>(cv, pl.scalpow, lane, [] { __syncwarp(); });
    for (int q = 0; q < ntile; q++) {
        const uint64_t c = ct_index(rc, wfirst, q);
        uint32_t *erow = a.err ? a.err + (a.err_off ? a.err_off[c] : c * (uint64_t)a.err_stride) : nullptr;
        uint16_t *prow = a.pos ? a.pos + c * (uint64_t)a.pos_stride : nullptr;
        uint8_t *epack = a.err_packed ? a.err_packed + c * (uint64_t)(Set<S>::N / 8) : nullptr;
        const int cnt = fft_root_one<S, M>(cv, q, fa, pl.tw, rc.key.bctl, erow, prow, lane, epack);
        if (lane == 0 && a.weight)
            a.weight[c] = (uint16_t)cnt;
    }
}

template <int SETMASK, int WPB>
__global__ void __launch_bounds__(WPB * 32, 1) k_fused(FusedArgs a)
{
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t s_round;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            s_round = atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const uint32_t r = s_round;
        if (r >= a.ntiles)
            return;
        RoundCtx rc;
        rc.a = &a;
        if (a.tiles) {
            rc.tile = a.tiles[r];
            rc.key = a.keys[rc.tile.key];
        } else {
            const uint64_t first = (uint64_t)r * a.round_cts;
            const uint64_t left = a.total - first;
            rc.tile = FusedTile{0u, (uint32_t)(left < a.round_cts ? left : a.round_cts), first};
            rc.key = a.key0;
        }
        const int set = a.single_set >= 0 ? a.single_set : rc.key.set;
        if ((SETMASK & (1 << S348864)) && set == S348864)
            fused_round<S348864, WPB>(rc, smem);
        else if ((SETMASK & (1 << S460896)) && set == S460896)
            fused_round<S460896, WPB>(rc, smem);
        else if ((SETMASK & (1 << S6688128)) && set == S6688128)
            fused_round<S6688128, WPB>(rc, smem);
        else if ((SETMASK & (1 << S6960119)) && set == S6960119)
            fused_round<S6960119, WPB>(rc, smem);
        else if ((SETMASK & (1 << S8192128)) && set == S8192128)
            fused_round<S8192128, WPB>(rc, smem);
    }
}

template <int S> constexpr size_t fz_smem(int wpb) { return (size_t)Fz<S>::SYN_B + (size_t)wpb * Fz<S>::WARP_B; }

size_t smem_limit_bytes();

// Per-instantiation launch and occupancy helpers (one translation unit per
// set mask, so the instantiations compile in parallel).
// Raises the kernel's dynamic shared-memory limit to `smem` (never lowers
// it; the opt-in maximum per CTA includes the kernel's static shared memory,
// so the attribute is set to what a launch needs, not to the device limit).
template <int SETMASK, int WPB> cudaError_t ensure_smem_attr(size_t smem)
{
    static size_t given[64] = {};  // per device: the attribute is a per-device setting
    int dev = 0;
    cudaGetDevice(&dev);
    size_t &set_to = given[dev & 63];
    if (smem <= set_to)
        return cudaSuccess;
    cudaError_t e =
        cudaFuncSetAttribute(k_fused<SETMASK, WPB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        set_to = smem;
    return e;
}

template <int SETMASK, int WPB> cudaError_t launch_k(const FusedArgs &a, int grid, size_t smem, cudaStream_t s)
{
    cudaError_t e = ensure_smem_attr<SETMASK, WPB>(smem);
    if (e != cudaSuccess)
        return e;
    k_fused<SETMASK, WPB><<<grid, WPB * 32, smem, s>>>(a);
    return cudaGetLastError();
}

template <int SETMASK, int WPB> int occupancy(size_t smem)
{
    if (ensure_smem_attr<SETMASK, WPB>(smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_fused<SETMASK, WPB>, WPB * 32, smem) != cudaSuccess)
        return 1;
    return n;
}

// Entry points defined in fused_m<mask>.cu.
#define CMD_FUSED_DECL(MASK)                                                              \
    cudaError_t fused_launch_##MASK(const FusedArgs &a, int grid, int wpb, size_t smem, cudaStream_t s); \
    int fused_occ_##MASK(int wpb, size_t smem);
CMD_FUSED_DECL(1)
CMD_FUSED_DECL(2)
CMD_FUSED_DECL(4)
CMD_FUSED_DECL(8)
CMD_FUSED_DECL(16)
CMD_FUSED_DECL(31)
#undef CMD_FUSED_DECL

}  // namespace cmd
