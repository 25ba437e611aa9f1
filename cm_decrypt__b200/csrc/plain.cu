// Plain per-stage decrypt path: three kernels, one per reference stage, with
// the intermediate syndromes and locators in global memory.
//   k_synd_plain  -- synd()   (CPU/param/param6960119/src/util.c:102-114)
//   k_bm_plain    -- bm()     (CPU/src/common/bm.c:12-68)
//   k_root_plain  -- root() + build_error_vector (root_13.c:233-240,
//                    decrypt.c:43-53), with the weight count fused in
#include "gf.cuh"
#include "internal.h"

namespace cmd {

constexpr uint32_t FULL = 0xFFFFFFFFu;

// ---------------------------------------------------------------- syndrome
// One warp per ciphertext, 8 per CTA.  The CTA stages its 8 ciphertexts and
// then 32-row chunks of the syndrome table in shared memory with 128-bit
// loads, so each table chunk read from L2 serves 8 ciphertexts.  Lane l
// accumulates table words l, l+32, ... of every row whose ciphertext bit is
// set; the bit is turned into an all-ones/zero mask (no data-dependent
// branch).  Output row = t words = the 2t syndromes as u16 pairs.
constexpr int SYND_CPB = 8, SYND_ROWS = 32;

template <int S> __global__ void __launch_bounds__(256) k_synd_plain(const uint32_t *__restrict__ tab,
                                                                     const uint8_t *__restrict__ cts,
                                                                     size_t count, uint32_t *__restrict__ synd)
{
    using P = Set<S>;
    constexpr int TW = P::TW, TWP = P::TWP, KW = (TW + 31) / 32;
    constexpr int RAW = SYND_CPB * P::CT;  // multiple of 16 bytes for every set
    __shared__ __align__(16) uint8_t s_ct[RAW];
    __shared__ __align__(16) uint32_t s_tab[SYND_ROWS * TWP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t c0 = (size_t)blockIdx.x * SYND_CPB;
    const size_t nct = count - c0 < (size_t)SYND_CPB ? count - c0 : SYND_CPB;

    {   // stage the ciphertexts: full groups are 16-byte aligned slabs
        const uint8_t *src = cts + c0 * P::CT;
        const int bytes = (int)nct * P::CT;
        if (bytes == RAW && (((uintptr_t)src) & 15) == 0) {
            for (int v = threadIdx.x; v < RAW / 16; v += blockDim.x)
                reinterpret_cast<uint4 *>(s_ct)[v] = reinterpret_cast<const uint4 *>(src)[v];
        } else {
            for (int v = threadIdx.x; v < RAW; v += blockDim.x)
                s_ct[v] = v < bytes ? src[v] : 0;
        }
    }
    uint32_t acc[KW];
#pragma unroll
    for (int k = 0; k < KW; k++)
        acc[k] = 0;
    const uint8_t *my_ct = s_ct + warp * P::CT;

    for (int b0 = 0; b0 < P::SB; b0 += SYND_ROWS) {
        const int rows = P::SB - b0 < SYND_ROWS ? P::SB - b0 : SYND_ROWS;
        __syncthreads();
        // rows are TWP (multiple of 4) words, so every chunk is 16-byte aligned
        const uint32_t *src = tab + (size_t)b0 * TWP;
        const int words = rows * TWP;
        for (int v = threadIdx.x; v < words / 4; v += blockDim.x)
            reinterpret_cast<uint4 *>(s_tab)[v] = __ldg(reinterpret_cast<const uint4 *>(src) + v);
        __syncthreads();
        for (int r = 0; r < rows; r++) {
            const int b = b0 + r;
            const uint32_t mask = 0u - ((my_ct[b >> 3] >> (b & 7)) & 1u);
#pragma unroll
            for (int k = 0; k < KW; k++) {
                const int w = lane + 32 * k;
                if (w < TW)
                    acc[k] ^= s_tab[r * TWP + w] & mask;
            }
        }
    }
    if ((size_t)warp < nct) {
        uint32_t *out = synd + (c0 + warp) * TW;
#pragma unroll
        for (int k = 0; k < KW; k++) {
            const int w = lane + 32 * k;
            if (w < TW)
                out[w] = acc[k];
        }
    }
}

// --------------------------------------------------------- Berlekamp-Massey
// One warp per ciphertext.  Lane l owns coefficients i = l + 32j of C and B
// in registers.  The discrepancy is a shuffle-XOR reduction of the lanes'
// partial sums; x*B moves each coefficient one lane up (lane 0 takes lane
// 31's previous slot).  Semantics follow bm.c exactly: t+1 coefficients, the
// discrepancy sums i <= min(N,t), B[t] is dropped by the shift, and the
// output is reversed (out[i] = C[t-i]).  Update decisions are masks.
template <int S> __global__ void __launch_bounds__(256) k_bm_plain(const uint16_t *__restrict__ synd, size_t count,
                                                                   uint16_t *__restrict__ loc)
{
    using P = Set<S>;
    constexpr int M = P::M, T = P::T, NJ = (T + 1 + 31) / 32;
    __shared__ uint16_t s_s[8][2 * T];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t c = (size_t)blockIdx.x * 8 + warp;
    if (c >= count)
        return;  // whole warp leaves together
    for (int j = lane; j < 2 * T; j += 32)
        s_s[warp][j] = synd[c * 2 * T + j];
    __syncwarp();
    const uint16_t *s = s_s[warp];

    uint32_t C[NJ], B[NJ];
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const int i = lane + 32 * j;
        C[j] = (i == 0);
        B[j] = (i == 1);
    }
    // f = d/b = d * b^-1 (gf_frac's value): b changes only when L does, so
    // b^-1 is kept and inverted again only then, off the next discrepancy's
    // path (bm.c recomputes gf_frac(b, d) every step).
    uint32_t b = 1, binv = 1, L = 0;
    for (int N = 0; N < 2 * T; N++) {
        // deg C <= L: coefficients above L are zero and add nothing to the
        // discrepancy (bm.c sums i <= min(N, t); the terms above L vanish)
        const int lim = min(N < T ? N : T, (int)L);
        uint32_t part = 0;
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int i = lane + 32 * j;
            if (32 * j <= lim && i <= lim)
                part ^= gf_mul<M>(C[j], s[N - i]);
        }
        const uint32_t d = __reduce_xor_sync(FULL, part);
        const uint32_t mne = 0u - (uint32_t)(d != 0);
        const uint32_t mle = mne & (0u - (uint32_t)((uint32_t)N >= 2 * L));
        const uint32_t f = gf_mul<M>(d, binv);
        const uint32_t Ln = (L & ~mle) | ((N + 1 - L) & mle);
        const int ub = min((int)Ln, T);  // the new C is zero above the new L
        uint32_t sel[NJ];
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const uint32_t oc = C[j];
            if (32 * j <= ub)
                C[j] ^= gf_mul<M>(f, B[j]) & mne;
            sel[j] = (B[j] & ~mle) | (oc & mle);
        }
        L = Ln;
        b = (b & ~mle) | (d & mle);
        if (mle)  // the same for the whole warp: one ciphertext
            binv = gf_inv<M>(d);
        uint32_t up[NJ];
#pragma unroll
        for (int j = 0; j < NJ; j++)
            up[j] = __shfl_sync(FULL, sel[j], (lane + 31) & 31);
#pragma unroll
        for (int j = 0; j < NJ; j++) {
            const int i = lane + 32 * j;
            const uint32_t nb = lane == 0 ? (j == 0 ? 0u : up[j > 0 ? j - 1 : 0]) : up[j];
            B[j] = i <= T ? nb : 0u;
        }
    }
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        const int i = lane + 32 * j;
        if (i <= T)
            loc[c * (T + 1) + (T - i)] = (uint16_t)C[j];
    }
}

// -------------------------------------------------------------- root search
// Bitsliced Horner: thread w owns support word w (32 points; its m planes
// stay in registers for every ciphertext the CTA processes).  Per ciphertext
// the CTA expands the t+1 locator coefficients into all-ones/zero plane masks
// in shared memory, then every thread runs t steps of r <- r*a + f[i] on its
// 32 points at once.  A point is a root iff all m planes of r are zero there:
// that word is directly the packed error-vector word.  The weight (flagged
// positions) is reduced across the CTA.
template <int S> constexpr int root_threads() { return ((Set<S>::NW + 31) / 32) * 32; }

template <int S>
__global__ void __launch_bounds__(root_threads<S>()) k_root_plain(const uint32_t *__restrict__ Lbs,
                                                                  const uint16_t *__restrict__ loc, size_t count,
                                                                  uint32_t *__restrict__ err,
                                                                  uint16_t *__restrict__ weight)
{
    using P = Set<S>;
    constexpr int M = P::M, T = P::T, NW = P::NW;
    constexpr int NWARP = root_threads<S>() / 32;
    __shared__ __align__(16) uint32_t s_mask[T + 1][16];
    __shared__ int s_cnt[NWARP];
    const int w = threadIdx.x, lane = w & 31, warp = w >> 5;
    uint32_t a[M];
#pragma unroll
    for (int k = 0; k < M; k++)
        a[k] = w < NW ? __ldg(Lbs + k * NW + w) : 0u;
    const int left = P::N - 32 * w;
    const uint32_t valid = w >= NW ? 0u : (left >= 32 ? FULL : ((1u << left) - 1u));

    for (size_t c = blockIdx.x; c < count; c += gridDim.x) {
        __syncthreads();
        const uint16_t *f = loc + c * (T + 1);
        for (int e = threadIdx.x; e < (T + 1) * 16; e += blockDim.x) {
            const int i = e >> 4, k = e & 15;
            s_mask[i][k] = k < M ? 0u - ((uint32_t)(__ldg(f + i) >> k) & 1u) : 0u;
        }
        __syncthreads();
        uint32_t r[M];
#pragma unroll
        for (int k = 0; k < M; k++)
            r[k] = s_mask[T][k];
        for (int i = T - 1; i >= 0; i--) {
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
        const uint32_t z = ~any & valid;
        if (w < NW)
            err[c * NW + w] = z;
        int cnt = __popc(z);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            cnt += __shfl_xor_sync(FULL, cnt, off);
        if (lane == 0)
            s_cnt[warp] = cnt;
        __syncthreads();
        if (w == 0 && weight) {
            int tot = 0;
#pragma unroll
            for (int q = 0; q < NWARP; q++)
                tot += s_cnt[q];
            weight[c] = (uint16_t)tot;
        }
    }
}

// Scalar images f(L_i) for stage-level parity tests (not on the hot path).
template <int S> __global__ void __launch_bounds__(256) k_root_images(const uint16_t *__restrict__ L,
                                                                      const uint16_t *__restrict__ loc, size_t count,
                                                                      uint16_t *__restrict__ images)
{
    using P = Set<S>;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= count * P::N)
        return;
    const size_t c = idx / P::N;
    const int i = (int)(idx % P::N);
    const uint16_t *f = loc + c * (P::T + 1);
    const uint32_t a = L[i];
    uint32_t r = f[P::T];
    for (int j = P::T - 1; j >= 0; j--)
        r = gf_mul<P::M>(r, a) ^ f[j];
    images[idx] = (uint16_t)r;
}

// ------------------------------------------------------------------ launch

cudaError_t launch_synd_plain(const KeyDev &k, const uint8_t *d_cts, size_t count, uint32_t *d_synd,
                              cudaStream_t s, LaunchCounter lc)
{
    if (count == 0)
        return cudaSuccess;
    return dispatch_set(k.set, [&]<int S>() -> cudaError_t {
        const unsigned grid = (unsigned)((count + SYND_CPB - 1) / SYND_CPB);
        k_synd_plain<S><<<grid, 256, 0, s>>>(k.tab, d_cts, count, d_synd);
        lc.bump();
        return cudaGetLastError();
    });
}

cudaError_t launch_bm_plain(int set, const uint16_t *d_synd, size_t count, uint16_t *d_loc, cudaStream_t s,
                            LaunchCounter lc)
{
    if (count == 0)
        return cudaSuccess;
    return dispatch_set(set, [&]<int S>() -> cudaError_t {
        const unsigned grid = (unsigned)((count + 7) / 8);
        k_bm_plain<S><<<grid, 256, 0, s>>>(d_synd, count, d_loc);
        lc.bump();
        return cudaGetLastError();
    });
}

cudaError_t launch_root_plain(const KeyDev &k, const uint16_t *d_loc, size_t count, uint32_t *d_err,
                              uint16_t *d_weight, cudaStream_t s, LaunchCounter lc, int num_sms)
{
    if (count == 0)
        return cudaSuccess;
    return dispatch_set(k.set, [&]<int S>() -> cudaError_t {
        int per_sm = 1;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_root_plain<S>, root_threads<S>(), 0);
        size_t grid = (size_t)(per_sm > 0 ? per_sm : 1) * (size_t)num_sms;
        if (grid > count)
            grid = count;
        k_root_plain<S><<<(unsigned)grid, root_threads<S>(), 0, s>>>(k.Lbs, d_loc, count, d_err, d_weight);
        lc.bump();
        return cudaGetLastError();
    });
}

// Loads the plain kernels' module on the current device now (with lazy
// module loading, the default, a kernel's module is otherwise loaded, and its
// memory allocated, by its first launch).
cudaError_t preload_plain_kernels()
{
    cudaError_t e = cudaSuccess;
    auto one = [&](const void *f) {
        cudaFuncAttributes fa;
        if (e == cudaSuccess)
            e = cudaFuncGetAttributes(&fa, f);
    };
    for (int set = 0; set < NSETS; set++)
        dispatch_set(set, [&]<int S>() {
            one((const void *)k_synd_plain<S>);
            one((const void *)k_bm_plain<S>);
            one((const void *)k_root_plain<S>);
            return 0;
        });
    return e;
}

cudaError_t launch_root_images(const KeyDev &k, const uint16_t *d_loc, size_t count, uint16_t *d_images,
                               cudaStream_t s, LaunchCounter lc)
{
    if (count == 0)
        return cudaSuccess;
    return dispatch_set(k.set, [&]<int S>() -> cudaError_t {
        const size_t total = count * (size_t)Set<S>::N;
        k_root_images<S><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(k.L, d_loc, count, d_images);
        lc.bump();
        return cudaGetLastError();
    });
}

}  // namespace cmd
