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
// k_tile_bm: one CTA of 8 warps per tile.
//   1. syndrome: warp w computes ciphertexts 4w..4w+3; lane l owns table words
//      4l..4l+3 (one 128-bit load per row from the ciphertext's key table),
//      every row masked by the ciphertext bit;
//   2. ballot transpose to bitsliced syndromes (bit q = ciphertext q);
//   3. scaled Berlekamp-Massey bitsliced across the 32 ciphertexts with thread
//      i owning coefficient i, so one step costs about one bitsliced multiply
//      per thread: partial discrepancies meet in shared memory, B lives in a
//      shared ring buffer whose rotation is the x*B shift;
//   4. the bitsliced locator (t+1 coefficients x 16 words) goes to global.
// k_root_tile: one CTA per ciphertext, bitsliced Horner over its support.
constexpr int TILE_LOC_WORDS = 130 * 16;

template <int S> struct TileSmem {
    using P = Set<S>;
    static constexpr int SYN_STRIDE = P::TW | 1;  // odd stride: conflict-free column reads
    uint8_t ct[32][(P::CT + 15) / 16 * 16];
    uint32_t syn[32 * SYN_STRIDE];
    uint32_t S_[2 * P::T * P::M];
    uint32_t ring[(P::T + 2) * P::M];
    uint32_t part[2][8][16];  // per-warp partial discrepancies, double-buffered by step parity
};

template <int S> __device__ __forceinline__ void tile_bm(const LatItem *items, int count, const uint8_t *cts,
                                                         uint32_t *loc_bs, uint8_t *smem_raw)
{
    using P = Set<S>;
    using Sm = TileSmem<S>;
    constexpr int M = P::M, T = P::T, TW = P::TW, TWP = P::TWP, R = T + 2;
    constexpr int NWB = (T + 1 + 31) / 32;  // warps that own coefficients
    constexpr int SYN = Sm::SYN_STRIDE;
    Sm &sm = *reinterpret_cast<Sm *>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // ---- 1. syndromes, four ciphertexts at a time -------------------------
    // All 8 warps work on each group of 4, warp w taking table rows w, w+8,
    // ...: a lone ciphertext gets the whole CTA's memory parallelism (its
    // key's table is usually in HBM, not L2).  Lane l owns table words
    // 4l..4l+3 (one 128-bit load per row); partial syndromes meet in shared
    // memory by XOR.
    for (int v = tid; v < 32 * P::CT; v += blockDim.x) {
        const int q = v / P::CT, o = v - q * P::CT;
        sm.ct[q][o] = q < count ? cts[items[q].ct_off + o] : 0;
    }
    for (int v = tid; v < 32 * SYN; v += blockDim.x)
        sm.syn[v] = 0;
    __syncthreads();
    const bool live = 4 * lane < TWP;
    for (int g = 0; 4 * g < count; g++) {
        const uint32_t *tab[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int q = 4 * g + u;
            tab[u] = items[q < count ? q : 0].tab;
        }
        uint4 acc[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
            acc[u] = make_uint4(0, 0, 0, 0);
#pragma unroll 4
        for (int b = warp; b < P::SB; b += 8) {
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const uint32_t m = 0u - ((sm.ct[4 * g + u][b >> 3] >> (b & 7)) & 1u);
                if (live) {
                    const uint4 x = __ldg(reinterpret_cast<const uint4 *>(tab[u] + (size_t)b * TWP) + lane);
                    acc[u].x ^= x.x & m;
                    acc[u].y ^= x.y & m;
                    acc[u].z ^= x.z & m;
                    acc[u].w ^= x.w & m;
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int q = 4 * g + u;
            const uint32_t v4[4] = {acc[u].x, acc[u].y, acc[u].z, acc[u].w};
#pragma unroll
            for (int e = 0; e < 4; e++)
                if (q < count && 4 * lane + e < TW)
                    atomicXor(&sm.syn[q * SYN + 4 * lane + e], v4[e]);
        }
    }
    __syncthreads();

    // ---- 2. transpose: S_[j*M + k] bit q = bit k of syndrome j of ct q ----
    for (int w = warp; w < TW; w += 8) {
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

    // ---- 3. scaled Berlekamp-Massey, thread i owns coefficient i ----------
    // One barrier per step: right after updating its coefficient a thread
    // already computes its share of the next step's discrepancy.
    const int i = tid;
    uint32_t C[M], bb[M];
#pragma unroll
    for (int k = 0; k < M; k++) {
        C[k] = (i == 0 && k == 0) ? FULL : 0u;
        bb[k] = k == 0 ? FULL : 0u;
    }
    int Lq = 0;  // L of ciphertext `lane` (every warp keeps a copy)
    // share of discrepancy N (N = 0 here): C_i * S_{N-i} for i <= min(N, t),
    // XOR-reduced over the warp into part[warp]
    auto partial = [&](int N) {
        if (warp >= NWB)
            return;
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
    partial(0);
    __syncthreads();
#pragma unroll 1
    for (int N = 0; N < 2 * T; N++) {
        uint32_t d[M], mne = 0;
#pragma unroll
        for (int k = 0; k < M; k++) {
            uint32_t v = 0;
#pragma unroll
            for (int w = 0; w < NWB; w++)
                v ^= sm.part[N & 1][w][k];
            d[k] = v;
            mne |= v;
        }
        const bool my_mle = ((mne >> lane) & 1u) && (N >= 2 * Lq);
        const uint32_t mle = __ballot_sync(FULL, my_mle);
        Lq = my_mle ? N + 1 - Lq : Lq;
        if (i <= T) {
            int slot = i + (R - (N % R)) % R;
            slot = slot >= R ? slot - R : slot;
            uint32_t *bp = sm.ring + slot * M;
            uint32_t bv[M], q[2 * M - 1];
#pragma unroll
            for (int k = 0; k < M; k++)
                bv[k] = bp[k];
#pragma unroll
            for (int k = 0; k < 2 * M - 1; k++)
                q[k] = 0;
            bs_mul_acc<M>(q, bb, C);
            bs_mul_acc<M>(q, d, bv);
            bs_reduce<M>(q);
#pragma unroll
            for (int k = 0; k < M; k++) {
                bp[k] = (bv[k] & ~mle) | (C[k] & mle);
                C[k] = q[k];
            }
        }
        const int freeslot = (R - ((N + 1) % R)) % R;
        if (tid < M)
            sm.ring[freeslot * M + tid] = 0;
#pragma unroll
        for (int k = 0; k < M; k++)
            bb[k] = (bb[k] & ~mle) | (d[k] & mle);
        if (N + 1 < 2 * T)
            partial(N + 1);  // writes part[(N+1)&1]; part[N&1] was read above
        __syncthreads();
    }
    // ---- 4. bitsliced locator out -----------------------------------------
    if (i <= T)
#pragma unroll
        for (int k = 0; k < M; k++)
            loc_bs[i * 16 + k] = C[k];
}

__global__ void __launch_bounds__(256) k_tile_bm(const LatItem *__restrict__ items, const uint8_t *__restrict__ cts,
                                                 uint32_t *__restrict__ loc_bs)
{
    extern __shared__ __align__(16) uint8_t smem_tile[];
    const LatItem *ti = items + (size_t)blockIdx.x * 32;
    const int count = (int)ti[0].pad;
    uint32_t *out = loc_bs + (size_t)blockIdx.x * TILE_LOC_WORDS;
    switch (ti[0].set) {
    case S348864: tile_bm<S348864>(ti, count, cts, out, smem_tile); break;
    case S460896: tile_bm<S460896>(ti, count, cts, out, smem_tile); break;
    case S6688128: tile_bm<S6688128>(ti, count, cts, out, smem_tile); break;
    case S6960119: tile_bm<S6960119>(ti, count, cts, out, smem_tile); break;
    default: tile_bm<S8192128>(ti, count, cts, out, smem_tile); break;
    }
}

template <int S> __device__ __forceinline__ void root_tile(const LatItem &it, const uint32_t *loc_tile, int q,
                                                           uint32_t *err, uint16_t *weight, uint32_t (*s_mask)[16],
                                                           int *s_cnt)
{
    using P = Set<S>;
    constexpr int M = P::M, T = P::T, NW = P::NW;
    const int w = threadIdx.x, lane = w & 31, warp = w >> 5;
    for (int e = threadIdx.x; e < (T + 1) * 16; e += blockDim.x) {
        const int i = e >> 4, k = e & 15;
        s_mask[i][k] = k < M ? 0u - ((loc_tile[i * 16 + k] >> q) & 1u) : 0u;
    }
    uint32_t a[M];
#pragma unroll
    for (int k = 0; k < M; k++)
        a[k] = w < NW ? __ldg(it.Lbs + k * NW + w) : 0u;
    __syncthreads();
    uint32_t r[M];
#pragma unroll
    for (int k = 0; k < M; k++)
        r[k] = s_mask[0][k];  // C[0] = f[t]
    for (int i = 1; i <= T; i++) {
        uint32_t p[2 * M - 1];
#pragma unroll
        for (int k = 0; k < 2 * M - 1; k++)
            p[k] = k < M ? s_mask[i][k] : 0u;
        bs_mul_acc<M>(p, r, a);
        bs_reduce<M>(p);
#pragma unroll
        for (int k = 0; k < M; k++)
            r[k] = p[k];
    }
    uint32_t any = 0;
#pragma unroll
    for (int k = 0; k < M; k++)
        any |= r[k];
    const int left = P::N - 32 * w;
    const uint32_t valid = w >= NW ? 0u : (left >= 32 ? FULL : ((1u << left) - 1u));
    const uint32_t z = ~any & valid;
    if (w < NW)
        err[it.err_off + w] = z;
    int cnt = __popc(z);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
        cnt += __shfl_xor_sync(FULL, cnt, off);
    if (lane == 0)
        s_cnt[warp] = cnt;
    __syncthreads();
    if (w == 0 && weight) {
        int tot = 0;
        for (int qq = 0; qq < 8; qq++)
            tot += s_cnt[qq];
        *weight = (uint16_t)tot;
    }
}

__global__ void __launch_bounds__(256) k_root_tile(const LatItem *__restrict__ items,
                                                   const uint32_t *__restrict__ loc_bs, uint32_t *__restrict__ err,
                                                   uint16_t *__restrict__ weight)
{
    __shared__ __align__(16) uint32_t s_mask[129][16];
    __shared__ int s_cnt[8];
    const int slot = blockIdx.x, t = slot >> 5, q = slot & 31;
    const LatItem it = items[slot];
    if (it.set < 0 || q >= (int)items[(size_t)t * 32].pad)
        return;
    const uint32_t *lt = loc_bs + (size_t)t * TILE_LOC_WORDS;
    uint16_t *wp = weight ? weight + slot : nullptr;
    switch (it.set) {
    case S348864: root_tile<S348864>(it, lt, q, err, wp, s_mask, s_cnt); break;
    case S460896: root_tile<S460896>(it, lt, q, err, wp, s_mask, s_cnt); break;
    case S6688128: root_tile<S6688128>(it, lt, q, err, wp, s_mask, s_cnt); break;
    case S6960119: root_tile<S6960119>(it, lt, q, err, wp, s_mask, s_cnt); break;
    default: root_tile<S8192128>(it, lt, q, err, wp, s_mask, s_cnt); break;
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
cudaError_t launch_tile_path(const void *d_items, const uint8_t *d_cts, uint32_t ntiles, uint32_t *d_loc_bs,
                             uint32_t *d_err, uint16_t *d_weight, cudaStream_t s, LaunchCounter lc)
{
    if (ntiles == 0)
        return cudaSuccess;
    static size_t attr = 0;
    const size_t smem = tile_smem_bytes();
    if (attr < smem) {
        cudaError_t e = cudaFuncSetAttribute(k_tile_bm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return e;
        attr = smem;
    }
    const LatItem *items = static_cast<const LatItem *>(d_items);
    k_tile_bm<<<ntiles, 256, smem, s>>>(items, d_cts, d_loc_bs);
    k_root_tile<<<ntiles * 32, 256, 0, s>>>(items, d_loc_bs, d_err, d_weight);
    lc.bump(2);
    return cudaGetLastError();
}

}  // namespace cmd
