// Latency-oriented decrypt path for the serving loop: tiles of up to 32
// ciphertexts of one parameter set, each ciphertext with its own key, in two
// launches per batch (any mix of sets: one tile per 32 ciphertexts of a set).
//
// Scaled Berlekamp-Massey.  bm() (CPU/src/common/bm.c:12-68) updates
// C <- C + (d/b) x B, which needs b^-1 every iteration: a chain of ~16
// dependent field operations per step.  Here C <- b C + d x B instead, with
// the same decisions (d != 0, N >= 2L), the same truncation to t+1
// coefficients and the same B/b/L updates.  By induction C_here = lambda *
// C_ref with lambda a product of earlier (nonzero) b values, so the returned
// polynomial is a nonzero multiple of bm()'s output: it has exactly the same
// roots and the decrypt flags exactly the same positions, decode failures
// included.  (The per-stage hook cmd_stage_bm keeps bm()'s exact output.)
#include <algorithm>

#include "fft_root.cuh"
#include "gf.cuh"
#include "internal.h"

namespace cmd {

namespace {
constexpr uint32_t FULL = 0xFFFFFFFFu;
}

static_assert(sizeof(LatItem) == 32, "LatItem layout");

// ---------------------------------------------------------------- tile path
// Tiles of up to 32 ciphertexts of one set, each with its own key.  Item slot
// 32*t + q is ciphertext q of tile t (LatItem.pad = the tile's count, padding
// slots have set -1).
//
// k_tile_synd: SYN_PARTS CTAs per ciphertext, each over a contiguous quarter
//   of the syndrome-table rows of the ciphertext's own key (util.c:102-114):
//   warp w takes rows w, w+8, ...; lane l owns table words 4l..4l+3 (one
//   128-bit load per row), every row masked by the ciphertext bit; the eight
//   warps' sums meet in shared memory and the CTA writes one partial
//   syndrome row.  A batch's tables stream through every SM at once instead
//   of through one SM per tile.
// k_tile_bm: one CTA of 8 warps per tile.
//   1. syndromes: XOR of each ciphertext's SYN_PARTS partial rows;
//   2. ballot transpose to bitsliced syndromes (bit q = ciphertext q);
//   3. scaled Berlekamp-Massey bitsliced across the 32 ciphertexts with thread
//      i owning coefficient i, so one step costs about one bitsliced multiply
//      per thread: partial discrepancies meet in shared memory, B lives in a
//      shared ring buffer whose rotation is the x*B shift;
//   4. radix conversion of the 32 locators by the whole CTA (fft_root.cuh);
//      the converted array (2^D entries x 16 words) goes to global.
// k_root_tile: 8 warps per CTA, four CTAs per tile, warp = one ciphertext:
// additive-FFT evaluation and the ciphertext's own key's support network.

template <int S>
__device__ __forceinline__ void tile_synd(const LatItem &it, const uint8_t *cts, int part, uint32_t *out,
                                          uint32_t (*red)[SYN_ROWW], uint8_t *ct)
{
    using P = Set<S>;
    constexpr int TWP = P::TWP, RPP = (P::SB + SYN_PARTS - 1) / SYN_PARTS;
    static_assert(TWP <= SYN_ROWW, "partial syndrome row");
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int v = tid; v < P::CT; v += blockDim.x)
        ct[v] = cts[it.ct_off + v];
    __syncthreads();
    const int b0 = part * RPP, b1 = b0 + RPP < P::SB ? b0 + RPP : P::SB;
    const bool live = 4 * lane < TWP;
    const uint4 *tab = reinterpret_cast<const uint4 *>(it.tab) + lane;
    uint4 acc = make_uint4(0, 0, 0, 0);
    // Rows whose ciphertext bit is clear are skipped (the bit is the same for
    // the whole warp, so the branch does not diverge): about half the table
    // is read.  The ciphertext is public, so which rows are read reveals
    // nothing about the key or the error vector.
#pragma unroll 8
    for (int b = b0 + warp; b < b1; b += 8) {
        if (live && ((ct[b >> 3] >> (b & 7)) & 1u)) {
            const uint4 x = __ldg(tab + (size_t)b * (TWP / 4));
            acc.x ^= x.x;
            acc.y ^= x.y;
            acc.z ^= x.z;
            acc.w ^= x.w;
        }
    }
    if (live)
        *reinterpret_cast<uint4 *>(&red[warp][4 * lane]) = acc;
    __syncthreads();
    for (int w = tid; w < TWP; w += blockDim.x) {
        uint32_t v = 0;
#pragma unroll
        for (int k = 0; k < 8; k++)
            v ^= red[k][w];
        out[w] = v;
    }
}

__global__ void __launch_bounds__(256) k_tile_synd(const LatItem *__restrict__ items, const uint8_t *__restrict__ cts,
                                                   uint32_t *__restrict__ synp)
{
    __shared__ __align__(16) uint32_t red[8][SYN_ROWW];
    __shared__ uint8_t ct[208];
    const int slot = blockIdx.x / SYN_PARTS, part = blockIdx.x % SYN_PARTS, t = slot >> 5, q = slot & 31;
    const LatItem it = items[slot];
    if (it.set < 0 || q >= (int)items[(size_t)t * 32].pad)
        return;  // whole CTA
    uint32_t *out = synp + ((size_t)slot * SYN_PARTS + part) * SYN_ROWW;
    switch (it.set) {
    case S348864: tile_synd<S348864>(it, cts, part, out, red, ct); break;
    case S460896: tile_synd<S460896>(it, cts, part, out, red, ct); break;
    case S6688128: tile_synd<S6688128>(it, cts, part, out, red, ct); break;
    case S6960119: tile_synd<S6960119>(it, cts, part, out, red, ct); break;
    default: tile_synd<S8192128>(it, cts, part, out, red, ct); break;
    }
}

template <int S> struct TileSmem {
    using P = Set<S>;
    static constexpr int SYN_STRIDE = P::TW | 1;  // odd stride: conflict-free column reads
    uint32_t syn[32 * SYN_STRIDE];
    uint32_t S_[2 * P::T * P::M];
    uint32_t ring[(P::T + 2) * P::M];
    uint32_t cs[(P::T + 1) * P::M];       // C after each update, for the discrepancy warps
    alignas(16) uint32_t part[2][8][16];  // per-warp partial discrepancies, double-buffered by step parity
};

// Threads of k_tile_bm: two roles of up to five warps each (t+1 <= 129
// coefficients per role).  The kernel is bounded to 96 registers a thread
// so that two tiles share an SM: one tile keeps an SM's ALUs about half busy
// (its steps are a chain of dependent multiplies and barriers).
constexpr int TILE_THREADS = 320;

template <int S> __device__ __forceinline__ void tile_bm(int count, const uint32_t *synp, uint32_t *loc_bs,
                                                         const uint16_t *scalpow, uint8_t *smem_raw)
{
    using P = Set<S>;
    using Sm = TileSmem<S>;
    constexpr int M = P::M, T = P::T, TW = P::TW, R = T + 2;
    constexpr int NWB = (T + 1 + 31) / 32;  // warps that own coefficients
    constexpr int SYN = Sm::SYN_STRIDE;
    Sm &sm = *reinterpret_cast<Sm *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // ---- 1. syndromes: XOR of the partial rows from k_tile_synd ------------
    for (int v = tid; v < 32 * TW; v += blockDim.x) {
        const int q = v / TW, w = v - q * TW;
        uint32_t x = 0;
        if (q < count) {
            const uint32_t *src = synp + (size_t)q * SYN_PARTS * SYN_ROWW + w;
#pragma unroll
            for (int p = 0; p < SYN_PARTS; p++)
                x ^= src[p * SYN_ROWW];
        }
        sm.syn[q * SYN + w] = x;
    }
    __syncthreads();

    // ---- 2. transpose: S_[j*M + k] bit q = bit k of syndrome j of ct q ----
    for (int w = warp; w < TW; w += TILE_THREADS / 32) {
        const uint32_t v = sm.syn[lane * SYN + w];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int j = 2 * w + h;
#pragma unroll
            for (int k = 0; k < M; k++) {
                const uint32_t bal = __ballot_sync(FULL, (v >> (16 * h + k)) & 1u);
                if (lane == ((j * M + k) & 31))
                    sm.S_[j * M + k] = bal;
            }
        }
    }
    for (int v = tid; v < R * M; v += blockDim.x)
        sm.ring[v] = (v == M) ? FULL : 0u;  // B = x
    __syncthreads();

    // ---- 3. scaled Berlekamp-Massey, two warps per 32 coefficients ---------
    // Warps [NWB, 2 NWB) own the coefficients (thread i of the role owns C_i
    // and its B ring slot) and do the update C <- b*C + d*x*B; warps
    // [0, NWB) compute the shares C_i * S_{N-i} of the next discrepancy.
    // Per step: (A) update: d*x*B, the one product that needs this step's
    // discrepancy (b*C was formed in the previous step); barrier; (B) the
    // discrepancy warps multiply the new C by the syndromes while the
    // update warps form b*C for the next step; barrier.  Two warps per
    // scheduler share the work and hide each other's latency.
    const bool dsc = warp < NWB;
    const bool upd = warp >= NWB && warp < 2 * NWB;
    const int i = upd ? tid - 32 * NWB : tid;
    uint32_t C[M], bb[M], q1[2 * M - 1];
#pragma unroll
    for (int k = 0; k < M; k++) {
        C[k] = (i == 0 && k == 0) ? FULL : 0u;
        bb[k] = k == 0 ? FULL : 0u;
    }
#pragma unroll
    for (int k = 0; k < 2 * M - 1; k++)
        q1[k] = k < M ? C[k] : 0u;  // b*C with b = 1
    int Lq = 0;  // L of ciphertext `lane` (update warps)
    // discrepancy warps: share of discrepancy N, C_i * S_{N-i} for
    // i <= min(N, t), XOR-reduced over the warp into part[N & 1][warp]
    auto partial = [&](int N) {
        const int lim = N < T ? N : T;
        uint32_t p[2 * M - 1];
#pragma unroll
        for (int k = 0; k < 2 * M - 1; k++)
            p[k] = 0;
        if (i <= lim) {
            uint32_t s[M];
#pragma unroll
            for (int k = 0; k < M; k++)
                s[k] = sm.S_[(N - i) * M + k];
            bs_mul_acc<M>(p, C, s);
            bs_reduce<M>(p);
        }
#pragma unroll
        for (int k = 0; k < M; k++) {
            const uint32_t v = __reduce_xor_sync(FULL, p[k]);
            if (lane == 0)
                sm.part[N & 1][warp][k] = v;
        }
    };
    if (dsc)
        partial(0);
    __syncthreads();
#pragma unroll 1
    for (int N = 0; N < 2 * T; N++) {
        if (upd) {
            // (A) the discrepancy, then the update
            uint32_t dd[16];
#pragma unroll
            for (int k = 0; k < 16; k++)
                dd[k] = 0;
#pragma unroll
            for (int w = 0; w < NWB; w++) {
                const uint4 *pr = reinterpret_cast<const uint4 *>(sm.part[N & 1][w]);
#pragma unroll
                for (int v = 0; v < 4; v++) {
                    const uint4 x = pr[v];
                    dd[4 * v] ^= x.x;
                    dd[4 * v + 1] ^= x.y;
                    dd[4 * v + 2] ^= x.z;
                    dd[4 * v + 3] ^= x.w;
                }
            }
            uint32_t d[M], mne = 0;
#pragma unroll
            for (int k = 0; k < M; k++) {
                d[k] = dd[k];
                mne |= dd[k];
            }
            const bool my_mle = ((mne >> lane) & 1u) && (N >= 2 * Lq);
            const uint32_t mle = __ballot_sync(FULL, my_mle);
            Lq = my_mle ? N + 1 - Lq : Lq;
            // Coefficients above N + 1 of C and x*B are still zero (their
            // ring entries were never written): whole warps past that skip.
            if (i <= T && i <= N + 1) {
                int slot = i + (R - (N % R)) % R;
                slot = slot >= R ? slot - R : slot;
                uint32_t *bp = sm.ring + slot * M;
                uint32_t bv[M];
#pragma unroll
                for (int k = 0; k < M; k++)
                    bv[k] = bp[k];
                bs_mul_acc<M>(q1, d, bv);
                bs_reduce<M>(q1);
#pragma unroll
                for (int k = 0; k < M; k++) {
                    bp[k] = (bv[k] & ~mle) | (C[k] & mle);
                    C[k] = q1[k];
                    sm.cs[i * M + k] = q1[k];
                }
            }
            const int freeslot = (R - ((N + 1) % R)) % R;
            if (i < M)
                sm.ring[freeslot * M + i] = 0;
#pragma unroll
            for (int k = 0; k < M; k++)
                bb[k] = (bb[k] & ~mle) | (d[k] & mle);
        }
        __syncthreads();
        if (N + 1 < 2 * T) {
            // (B) next discrepancy shares; b*C for the next update
            if (dsc) {
                const int lim = N + 1 < T ? N + 1 : T;
                if (i <= lim)
#pragma unroll
                    for (int k = 0; k < M; k++)
                        C[k] = sm.cs[i * M + k];
                partial(N + 1);
            } else if (upd && i <= T && i <= N + 2) {
#pragma unroll
                for (int k = 0; k < 2 * M - 1; k++)
                    q1[k] = 0;
                bs_mul_acc<M>(q1, bb, C);
            }
            __syncthreads();
        }
    }
    // ---- 4. radix conversion, converted locators out -----------------------
    // Entry x of the conversion array is C[T-x] (bm.c:62-65 reverses the
    // locator before root() evaluates it), zero for T < x < 2^D; S_ is free.
    using F = FftDims<S>;
    static_assert(F::NX * M <= 2 * T * M && F::NX * 16 <= TILE_LOC_WORDS, "conversion array size");
    if (upd && i <= T)
#pragma unroll
        for (int k = 0; k < M; k++)
            sm.S_[(T - i) * M + k] = C[k];
    for (int v = tid; v < (F::NX - T - 1) * M; v += blockDim.x)
        sm.S_[(T + 1) * M + v] = 0u;
    __syncthreads();
    fft_convert<S, M, TILE_THREADS>(sm.S_, scalpow, tid, [] { __syncthreads(); });
    for (int v = tid; v < F::NX * M; v += blockDim.x) {
        const int x = v / M, k = v - x * M;
        loc_bs[x * 16 + k] = sm.S_[v];
    }
}

__global__ void __launch_bounds__(TILE_THREADS, 2) k_tile_bm(const LatItem *__restrict__ items, const uint32_t *__restrict__ synp,
                                                 uint32_t *__restrict__ loc_bs, FftPlans plans)
{
    extern __shared__ __align__(16) uint8_t smem_tile[];
    const LatItem *ti = items + (size_t)blockIdx.x * 32;
    const int count = (int)ti[0].pad;
    const uint32_t *sp = synp + (size_t)blockIdx.x * 32 * SYN_PARTS * SYN_ROWW;
    uint32_t *out = loc_bs + (size_t)blockIdx.x * TILE_LOC_WORDS;
    switch (ti[0].set) {
    case S348864: tile_bm<S348864>(count, sp, out, plans.p[S348864].scalpow, smem_tile); break;
    case S460896: tile_bm<S460896>(count, sp, out, plans.p[S460896].scalpow, smem_tile); break;
    case S6688128: tile_bm<S6688128>(count, sp, out, plans.p[S6688128].scalpow, smem_tile); break;
    case S6960119: tile_bm<S6960119>(count, sp, out, plans.p[S6960119].scalpow, smem_tile); break;
    default: tile_bm<S8192128>(count, sp, out, plans.p[S8192128].scalpow, smem_tile); break;
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
    const int cnt = fft_root_one<S, 16>(cv, q, fa, pl.tw, it.bctl, err + it.err_off, nullptr, lane);
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
    const uint32_t *cv = loc_bs + (size_t)t * TILE_LOC_WORDS;
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

// ntiles tiles of 32 item slots; weights are indexed by item slot.
cudaError_t launch_tile_path(const void *d_items, const uint8_t *d_cts, uint32_t ntiles, uint32_t *d_scratch,
                             uint32_t *d_err, uint16_t *d_weight, const FftPlans &plans, cudaStream_t s,
                             LaunchCounter lc)
{
    if (ntiles == 0)
        return cudaSuccess;
    // the opt-in is per device: remember what each device has been given
    static size_t attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    size_t &set_to = attr[dev & 63];
    const size_t smem = tile_smem_bytes();
    const size_t root_smem = ROOT_WARPS * ROOT_FA_WORDS * 4;
    if (set_to < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_tile_bm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_root_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)root_smem);
        // One shared-memory split for all three kernels, so that CTAs of
        // concurrent batches' kernels can share an SM without it draining to
        // change its split (two k_tile_bm or two k_root_tile CTAs per SM).
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_synd, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_bm, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_root_tile, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess)
            return e;
        set_to = smem;
    }
    const LatItem *items = static_cast<const LatItem *>(d_items);
    uint32_t *d_loc_bs = d_scratch;
    uint32_t *d_synp = d_scratch + (size_t)ntiles * TILE_LOC_WORDS;
    k_tile_synd<<<ntiles * 32 * SYN_PARTS, 256, 0, s>>>(items, d_cts, d_synp);
    k_tile_bm<<<ntiles, TILE_THREADS, smem, s>>>(items, d_synp, d_loc_bs, plans);
    k_root_tile<<<ntiles * 4, ROOT_WARPS * 32, root_smem, s>>>(items, d_loc_bs, d_err, d_weight, plans);
    lc.bump(3);
    return cudaGetLastError();
}

}  // namespace cmd
