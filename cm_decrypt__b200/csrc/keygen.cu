// On-device Classic McEliece key generation: crypto_kem_keypair of the
// reference's kem/ tree (kem/common/core/operations.c:36-107) for a batch of
// seeds, every stage on the GPU.  One attempt per pending key and round:
//
//  1. k_kg_expand     SHAKE256(64 || seed) -> r = s | perm | f | next seed,
//                     a chain of consecutive attempts per key (one warp per
//                     key, a Keccak-f[1600] state lane per thread)
//  2. k_kg_genpoly    minimal polynomial g of f in GF((2^m)^t): the powers
//                     f^0..f^t (even ones by squaring), then Gauss-Jordan
//                     over GF(2^m) (sk_gen.c:24-85); on the seed chains
//  3. k_kg_support    pi = indices ordered by their random words (bitonic
//                     sort of (word << 31 | index) in shared memory, rejected
//                     on equal words), L = bitrev(pi), 1/g(L), and the mt x n
//                     parity-check matrix, 32 columns per thread in bitsliced
//                     form (pk_gen.c:52-113)
//  4. elimination     blocked Gauss-Jordan on the first mt columns, 32 pivot
//                     columns per panel: k_ge_panel takes pivot rows from the
//                     rows not yet used, building a reduced basis of their
//                     panel words (a warp, 32 candidate rows at a time), and
//                     the 32 x 32 transform to the reduced pivot rows;
//                     k_ge_apply replaces the pivot rows by reduced ones and
//                     clears the panel columns of every other row.  Rows stay
//                     in place: a map gives the row holding each pivot.  The
//                     result is the unique reduced form [I | T] that
//                     pk_gen.c:115-143 reaches (rejected when a pivot is
//                     missing, i.e. the left block is singular)
//  5. k_kg_controlbits Benes control bits of pi by the cycle-labelling
//                     recursion (controlbits.c:22-170), all sub-networks of a
//                     level at once; the reference's sorts become the
//                     permutation inverses and compositions they compute.
//                     Checked by running the network (controlbits.c:180-220)
//  6. k_kg_output     pk rows (bytes mt/8 .. of each reduced row,
//                     pk_gen.c:145-146) and sk = seed | pivots | g | control
//                     bits | s (operations.c:60-100)
//
// A rejected attempt continues with the next seed from r, exactly as the
// reference's loop does, so a seed yields the reference's key pair.
//
// The same parity-check matrix (from an existing key's support and Goppa
// polynomial, k_kg_support_key), elimination and a column transpose
// (k_kg_pk_columns) give the public-key columns that decapsulation checks
// re-encodings against: kg_pubkey_columns.
//
// Not all constant-time.  All field arithmetic is table-free: the Goppa
// polynomial uses a multiply by integer multiplies on operands with holes and
// the inversion chain over it (its zero-pivot fix-up is a masked row sum), and the support stage (sort, L,
// g(L), 1/g(L), the parity-check matrix) is bitonic sorting plus the bitsliced
// routines.  The elimination reads the rows it chooses and indexes its
// combination tables by panel words, and the control-bit recursion indexes
// by permutation values, so those two stages' timing depends on secret
// values.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <vector>

#include "engine.h"
#include "gf.cuh"
#include "keccak.cuh"

namespace cmd {
namespace {

constexpr int KG_MAX_Q = 1 << 13;
constexpr int PANEL = 32;

enum KgStatus : int { KG_OK = 0, KG_GENPOLY = 1, KG_PERM = 2, KG_SINGULAR = 3, KG_CBITS = 4 };

// Runtime sizes of one set's key generation and the per-key workspace.
struct KgDims {
    int set, m, n, t, q, mt, rlen, rw, pk_row, cond, sk;
    size_t off_r, off_irr, off_pi, off_cond, off_panel, off_src, off_prow, off_used, off_mat, stride;
};

struct PanelInfo {
    int status;          // KgStatus of this key's attempt
    int npiv;            // pivot columns in the current panel
    int scan0;           // every row below it holds a pivot
    int pad;
    uint32_t src[PANEL];  // the rows chosen for this panel; row src[b] receives pivot b
    uint32_t T[PANEL];    // reduced pivot b = XOR over bits j of T[b] of (pre-panel) row src[j]
};

KgDims kg_dims(int set)
{
    const SetInfo si = set_info(set);
    KgDims d;
    d.set = set;
    d.m = si.m;
    d.n = si.n;
    d.t = si.t;
    d.q = 1 << si.m;
    d.mt = si.m * si.t;
    d.rlen = si.n / 8 + 4 * d.q + 2 * si.t + 32;
    d.rw = ((si.n + 31) / 32 + 3) / 4 * 4;  // row words, 16-byte rows
    d.pk_row = (si.n - d.mt + 7) / 8;
    d.cond = si.cond;
    d.sk = si.sk;
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    size_t o = 0;
    d.off_r = o;
    o = al(o + d.rlen);
    d.off_irr = o;
    o = al(o + 2 * (size_t)d.t);
    d.off_pi = o;
    o = al(o + 2 * (size_t)d.q);
    d.off_cond = o;
    o = al(o + d.cond);
    d.off_panel = o;
    o = al(o + sizeof(PanelInfo));
    d.off_src = o;  // copies of the panel's chosen rows
    o = al(o + (size_t)PANEL * d.rw * 4);
    d.off_prow = o;  // row holding pivot i
    o = al(o + (size_t)d.mt * 4);
    d.off_used = o;  // 1: the row already holds a pivot
    o = al(o + (size_t)d.mt);
    d.off_mat = o;
    o = al(o + (size_t)d.mt * d.rw * 4);
    d.stride = o;
    return d;
}

__device__ __forceinline__ uint32_t bitrev_m(uint32_t v, int m) { return __brev(v) >> (32 - m); }

// ---- 1. seed expansion ----------------------------------------------------
// Keccak-f[1600] with one state lane per thread of a warp (lane i = x + 5y,
// threads 25..31 shadow lane 0), two levels of warp shuffles a round:
//  1. the lanes of this thread's column (for its parity C[x]) and the three
//     lanes that pi moves to (x, y), (x + 1, y) and (x + 2, y), the row
//     neighbours chi combines;
//  2. the parities C[x0 - 1] .. C[x0 + 3], where x0, x0 + 1 and x0 + 2 are the
//     columns of those three lanes: theta's D for each of them.
// Each thread then applies theta, rho and chi to its three lanes itself, so
// pi and chi cost no further exchange.
struct WarpKeccak {
    int col[4];   // the other lanes of this thread's column
    int src[3];   // the lanes pi moves to (x, y), (x + 1, y), (x + 2, y)
    int rho[3];   // and their rotations mod 32
    bool half[3]; // rotations of 32 or more: the halves swap first
    int par[5];   // lanes holding C[x0 - 1], C[x0], .., C[x0 + 3]
    bool iota;
    __device__ WarpKeccak(int lane)
    {
        const int l = lane < 25 ? lane : 0;
        const int x = l % 5, y = l / 5;
#pragma unroll
        for (int k = 0; k < 4; k++)
            col[k] = x + 5 * ((y + 1 + k) % 5);
        // B[y, 2x + 3y] = A[x, y]: position (X, Y) takes lane (x0, y0) with
        // y0 = X and 2 x0 + 3 y0 = Y (mod 5), so x0 = 3 (Y - 3 X); position
        // (X + k, Y) takes (x0 + k, X + k)
        const int x0 = (3 * (((y - 3 * x) % 5 + 5) % 5)) % 5;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            src[k] = (x0 + k) % 5 + 5 * ((x + k) % 5);
            const int r = keccak_rot((x0 + k) % 5, (x + k) % 5);
            rho[k] = r & 31;
            half[k] = r >= 32;
        }
#pragma unroll
        for (int k = 0; k < 5; k++)
            par[k] = (x0 + 4 + k) % 5;  // lane q < 5 holds C[q]
        iota = l == 0;
    }
    // rotation by this thread's k-th offset: two funnel shifts on the halves
    __device__ __forceinline__ uint64_t rot(uint64_t v, int k) const
    {
        const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
        const uint32_t h = half[k] ? lo : hi, l = half[k] ? hi : lo;
        return ((uint64_t)__funnelshift_l(l, h, rho[k]) << 32) | __funnelshift_l(h, l, rho[k]);
    }
    __device__ uint64_t permute(uint64_t a) const
    {
        const unsigned F = 0xFFFFFFFFu;
#pragma unroll 1
        for (int round = 0; round < 24; round++) {
            uint64_t c = a;
#pragma unroll
            for (int k = 0; k < 4; k++)
                c ^= __shfl_sync(F, a, col[k]);
            const uint64_t a0 = __shfl_sync(F, a, src[0]), a1 = __shfl_sync(F, a, src[1]),
                           a2 = __shfl_sync(F, a, src[2]);
            const uint64_t cm1 = __shfl_sync(F, c, par[0]), c0 = __shfl_sync(F, c, par[1]),
                           c1 = __shfl_sync(F, c, par[2]), c2 = __shfl_sync(F, c, par[3]),
                           c3 = __shfl_sync(F, c, par[4]);
            // theta (D[x] = C[x - 1] ^ rotl(C[x + 1], 1)), then rho
            const uint64_t b0 = rot(a0 ^ cm1 ^ rotl64(c1, 1), 0);
            const uint64_t b1 = rot(a1 ^ c0 ^ rotl64(c2, 1), 1);
            const uint64_t b2 = rot(a2 ^ c1 ^ rotl64(c3, 1), 2);
            a = b0 ^ (~b1 & b2);  // chi
            if (iota)
                a ^= kRC[round];
        }
        return a;
    }
};

constexpr int SPEC = 4;  // attempts of one key expanded ahead (its chain)

// Warp k expands the next SPEC attempts of key keys[k] into its chain:
// attempt 0 from seeds[k] when given, else from the last 32 bytes of the
// key's previous chain entry Dprev - 1 (the seed the reference's loop moves
// on to after a rejected attempt); attempt j + 1 from attempt j's last 32
// bytes.  Chain entry j of key `out` is chain + (out * SPEC + j) * r_stride,
// its seed chain_seed + (out * SPEC + j) * 32.
__global__ void __launch_bounds__(32) k_kg_expand(const uint8_t *__restrict__ seeds, const int *__restrict__ keys,
                                                  uint8_t *__restrict__ chain, uint8_t *__restrict__ chain_seed,
                                                  KgDims d, int K, int Dprev, size_t r_stride)
{
    const int k = blockIdx.x, lane = threadIdx.x;
    if (k >= K)
        return;
    constexpr int RATE = 136;
    const WarpKeccak kc(lane);
    const int out = keys[k];
    uint8_t *base = chain + (size_t)out * SPEC * r_stride;
    // this lane's byte of the first seed, read before the chain is rewritten
    uint8_t sb = seeds ? seeds[(size_t)k * 32 + lane] : base[(size_t)(Dprev - 1) * r_stride + d.rlen - 32 + lane];
    __syncwarp();
    for (int j = 0; j < SPEC; j++) {
        uint8_t *r = base + (size_t)j * r_stride;
        chain_seed[((size_t)out * SPEC + j) * 32 + lane] = sb;
        // absorb 64 || seed || 0x1F, pad to 136 bytes with 0x80 at the end:
        // block byte i is 64 (i = 0), seed[i - 1] (1..32), 0x1F (33)
        uint64_t a = 0;
#pragma unroll
        for (int b = 0; b < 8; b++) {
            const int i = 8 * (lane < 5 ? lane : 0) + b;
            const uint32_t sv = __shfl_sync(0xFFFFFFFFu, (uint32_t)sb, (i - 1) & 31);
            uint32_t v = 0;
            if (i == 0)
                v = 64;
            else if (i <= 32)
                v = sv;
            else if (i == 33)
                v = 0x1F;
            if (lane < 5)
                a |= (uint64_t)v << (8 * b);
        }
        if (lane == 16)
            a ^= 0x8000000000000000ull;
        if (lane >= 25)
            a = 0;
#pragma unroll 1
        for (int off = 0; off < d.rlen; off += RATE) {
            a = kc.permute(a);
            const int len = min(RATE, d.rlen - off);
            if (lane < RATE / 8) {
                if (8 * lane + 8 <= len) {
                    reinterpret_cast<uint64_t *>(r + off)[lane] = a;  // r and off are 8-byte aligned
                } else if (8 * lane < len) {
                    for (int b = 0; b < len - 8 * lane; b++)
                        r[off + 8 * lane + b] = (uint8_t)(a >> (8 * b));
                }
            }
        }
        __syncwarp();  // the next attempt's seed is this one's last 32 bytes
        sb = r[d.rlen - 32 + lane];
        __syncwarp();
    }
}

// Slot k*D + j of the round takes chain entry j of key keys[k]: its
// expansion, its seed, its Goppa polynomial and status.
__global__ void k_kg_fill(const uint8_t *__restrict__ chain, const uint8_t *__restrict__ chain_seed,
                          const int *__restrict__ keys, uint8_t *__restrict__ work, uint8_t *__restrict__ slot_seed,
                          KgDims d, int D, size_t r_stride)
{
    const int slot = blockIdx.x, k = slot / D, j = slot - k * D, out = keys[k];
    const uint8_t *eb = chain + ((size_t)out * SPEC + j) * r_stride;
    const size_t r_al = (d.rlen + 255) / 256 * 256;
    uint8_t *wk = work + (size_t)slot * d.stride;
    const uint4 *src = reinterpret_cast<const uint4 *>(eb);
    uint4 *dst = reinterpret_cast<uint4 *>(wk + d.off_r);
    for (int i = threadIdx.x; i < (d.rlen + 15) / 16; i += blockDim.x)
        dst[i] = src[i];
    const uint16_t *gi = reinterpret_cast<const uint16_t *>(eb + r_al);
    uint16_t *go = reinterpret_cast<uint16_t *>(wk + d.off_irr);
    for (int i = threadIdx.x; i < d.t; i += blockDim.x)
        go[i] = gi[i];
    if (threadIdx.x < 32)
        slot_seed[(size_t)slot * 32 + threadIdx.x] = chain_seed[((size_t)out * SPEC + j) * 32 + threadIdx.x];
    if (threadIdx.x == 0)
        reinterpret_cast<PanelInfo *>(wk + d.off_panel)->status = *reinterpret_cast<const int *>(eb + r_al + 256);
}

// ---- 2. Goppa polynomial --------------------------------------------------
// Terms of F(y) = y^t + sum c_u y^off_u defining GF((2^m)^t)
// (kem/variant_<set>/gf.c GF_mul).
struct ExtPoly {
    int nt, off[4];
    uint16_t c[4];
};
__host__ __device__ inline ExtPoly ext_poly(int set)
{
    switch (set) {
    case S348864: return {3, {3, 1, 0, 0}, {1, 1, 2, 0}};        // y^64 + y^3 + y + z
    case S460896: return {4, {10, 9, 6, 0}, {1, 1, 1, 1}};       // y^96 + y^10 + y^9 + y^6 + 1
    case S6960119: return {2, {8, 0, 0, 0}, {1, 1, 0, 0}};       // y^119 + y^8 + 1
    default: return {4, {7, 2, 1, 0}, {1, 1, 1, 1}};             // y^128 + y^7 + y^2 + y + 1
    }
}

constexpr int GP_THREADS = 1024;

// Shared memory: the t x (t+1) system (row = coordinate, column = power),
// the current power, the product, the first fold, f, the multipliers and the
// pivot fix-up masks.
size_t genpoly_smem(const KgDims &d) { return (size_t)d.t * (d.t + 1) * 2 + 5 * 256 * 2 + 256 + 64; }

// One CTA per chain entry (key keys[blockIdx.x / SPEC], attempt
// blockIdx.x % SPEC): reads f from the entry's expansion, writes g and the
// attempt's status beside it.  Field arithmetic is table-free: the multiply
// by integer multiplies on operands with holes (gf_mul_im) and the inversion
// chain over it; memory addresses depend only on loop indices.
template <int M>
__device__ void genpoly_body(uint8_t *eb, uint8_t *smem, const KgDims &d, size_t r_al)
{
    uint16_t *A = reinterpret_cast<uint16_t *>(smem);  // [t][t+1]: row = coordinate, column = power
    uint16_t *pw = A + (size_t)d.t * (d.t + 1);       // 256: current power
    uint16_t *pr = pw + 256;                          // product, 2t - 1 <= 255
    uint16_t *v1 = pr + 256;                          // first fold, t + 10
    uint16_t *f = v1 + 256;                           // f
    uint16_t *col = f + 256;                          // multipliers of an elimination step
    uint8_t *add = reinterpret_cast<uint8_t *>(col + 256);  // rows added to fix a zero pivot
    __shared__ int s_ok;
    int *status = reinterpret_cast<int *>(eb + r_al + 256);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, t = d.t, W = t + 1;
    const uint8_t *fr = eb + d.rlen - 32 - 2 * t;
    if (tid < t) {
        f[tid] = (uint16_t)((fr[2 * tid] | (fr[2 * tid + 1] << 8)) & ((1u << M) - 1u));
        pw[tid] = tid == 0 ? 1 : 0;
    }
    __syncthreads();
    const ExtPoly F = ext_poly(d.set);
    int offmax = 0;
    for (int u = 0; u < F.nt; u++)
        offmax = max(offmax, F.off[u]);
    // powers f^0 .. f^t into the columns of A
    const int ko = tid >> 2, part = tid & 3;  // four threads per product coefficient
    for (int c = 0; c <= t; c++) {
        if (tid < t)
            A[tid * W + c] = pw[tid];
        if (c == t)
            break;
        __syncthreads();  // the squaring below may read column c itself (c = 1)
        if ((c + 1) % 2 == 0) {
            // f^(c+1) = (f^((c+1)/2))^2: squaring is linear in characteristic
            // 2 -- coefficient k squared lands at 2k (degree <= 2t - 2)
            if (tid < 2 * t - 1)
                pr[tid] = (tid & 1) ? 0 : (uint16_t)gf_sq<M>(A[(tid >> 1) * W + (c + 1) / 2]);
        } else {
            // pr = pw * f (degree <= 2t - 2)
            uint32_t acc = 0;
            if (ko < 2 * t - 1) {
                const int lo = max(0, ko - t + 1), hi = min(ko, t - 1);
                for (int i = lo + part; i <= hi; i += 4)
                    acc ^= gf_mul_im<M>(pw[i], f[ko - i]);
            }
            acc ^= __shfl_xor_sync(0xFFFFFFFFu, acc, 1);
            acc ^= __shfl_xor_sync(0xFFFFFFFFu, acc, 2);
            if (part == 0 && ko < 2 * t - 1)
                pr[ko] = (uint16_t)acc;
        }
        __syncthreads();
        // fold y^(t+i) = sum_u c_u y^(i+off_u): twice, the second for the at
        // most offmax coefficients the first pushes to degree >= t
        if (tid < t + offmax) {
            uint32_t acc = tid < t ? pr[tid] : 0;
            for (int u = 0; u < F.nt; u++) {
                const int i = tid - F.off[u];
                if (i >= 0 && i <= t - 2)
                    acc ^= gf_mul_im<M>(pr[t + i], F.c[u]);
            }
            v1[tid] = (uint16_t)acc;
        }
        __syncthreads();
        if (tid < t) {
            uint32_t acc = v1[tid];
            for (int u = 0; u < F.nt; u++) {
                const int i = tid - F.off[u];
                if (i >= 0 && i < offmax)
                    acc ^= gf_mul_im<M>(v1[t + i], F.c[u]);
            }
            pw[tid] = (uint16_t)acc;
        }
        __syncthreads();
    }
    __syncthreads();
    // Gauss-Jordan: sum_{j<t} g_j f^j = f^t.  A zero pivot is fixed as
    // sk_gen.c:46-53 does, by adding the following rows up to the first one
    // with a non-zero entry (masks from a prefix over the rows, no branch on
    // data); the pivot row is then scaled to 1 and cleared from the others.
    if (tid == 0)
        s_ok = 1;
    for (int c = 0; c < t; c++) {
        // add[k]: row k (> c) is added to row c -- when the pivot is zero,
        // rows c + 1 .. first (the first row with a non-zero entry in
        // column c); ballots over the rows, masks by comparison
        if (warp == 0) {
            int first = t;
            for (int base = c + 1; base < t; base += 32) {
                const int k = base + lane;
                const uint32_t bal = __ballot_sync(0xFFFFFFFFu, k < t && A[k * W + c] != 0);
                const int here = bal ? base + __ffs(bal) - 1 : t;
                first = first < t ? first : here;
            }
            const uint32_t zero = A[c * W + c] == 0;
            for (int k = c + 1 + lane; k < t; k += 32)
                add[k] = (uint8_t)(zero & (uint32_t)(k <= first));
            if (lane == 0)
                s_ok &= !(zero && first == t);  // no pivot: f's minimal polynomial has degree < t
        }
        __syncthreads();
        for (int x = c + tid; x <= t; x += GP_THREADS) {
            uint32_t acc = A[c * W + x];
            for (int k = c + 1; k < t; k++)
                acc ^= A[k * W + x] & (0u - (uint32_t)add[k]);
            A[c * W + x] = (uint16_t)acc;
        }
        __syncthreads();
        const uint32_t inv = gf_inv<M, true>(A[c * W + c]);  // 0 when singular (then s_ok = 0)
        __syncthreads();
        if (tid >= c && tid <= t)
            A[c * W + tid] = (uint16_t)gf_mul_im<M>(A[c * W + tid], inv);
        if (tid < t)
            col[tid] = tid == c ? 0 : A[tid * W + c];
        __syncthreads();
        for (int r = warp; r < t; r += GP_THREADS / 32) {
            const uint32_t k = col[r];
            for (int x = c + lane; x <= t; x += 32)
                A[r * W + x] ^= (uint16_t)gf_mul_im<M>(A[c * W + x], k);
        }
        __syncthreads();
    }
    uint16_t *irr = reinterpret_cast<uint16_t *>(eb + r_al);
    if (tid < t)
        irr[tid] = A[tid * W + t];
    if (tid == 0)
        *status = s_ok ? KG_OK : KG_GENPOLY;
}

__global__ void __launch_bounds__(GP_THREADS) k_kg_genpoly(uint8_t *__restrict__ chain, const int *__restrict__ keys,
                                                           KgDims d, size_t r_stride)
{
    extern __shared__ __align__(16) uint8_t sm_gp[];
    uint8_t *eb = chain + ((size_t)keys[blockIdx.x / SPEC] * SPEC + blockIdx.x % SPEC) * r_stride;
    const size_t r_al = (d.rlen + 255) / 256 * 256;
    if (d.m == 12)
        genpoly_body<12>(eb, sm_gp, d, r_al);
    else
        genpoly_body<13>(eb, sm_gp, d, r_al);
}

// ---- bitonic sorts in shared memory ----------------------------------------
// Ascending sort of each aligned segment of 2^seg_log elements of x[0, n)
// (n a power of two): the compare-exchange pattern depends on indices only.
template <class T>
__device__ void seg_sort(T *x, int n, int seg_log)
{
    const int seg = 1 << seg_log;
    for (int k = 2; k <= seg; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            __syncthreads();
            for (int p = threadIdx.x; p < n / 2; p += blockDim.x) {
                const int i = 2 * p - (p & (j - 1)), l = i + j;
                const bool asc = k == seg || !(i & k);
                const T a = x[i], b = x[l];
                const T lo = a < b ? a : b, hi = a < b ? b : a;
                x[i] = asc ? lo : hi;
                x[l] = asc ? hi : lo;
            }
        }
    }
    __syncthreads();
}

// ---- 3. support, 1/g(L) and the parity-check matrix ------------------------
constexpr int SUP_THREADS = 512;

// Shared memory: the sort buffer and g as bitsliced constants (t + 1 rows of
// 13 words).
size_t support_smem(const KgDims &d) { return (size_t)d.q * 8 + (size_t)(d.t + 1) * 13 * 4 + 16; }

// Columns 32 grp .. 32 grp + 31 of the parity-check matrix, bitsliced: L of
// the 32 columns as m plane words, g(L) by Horner, its inverse, then the
// rows L^j / g(L) -- plane word k of row j is the matrix word of row j*m + k.
// Multiplies and the inverse are the decrypt path's bitsliced routines:
// no tables, no data-dependent branch or index.
//
// The support comes from the sorted buffer (L = bitrev of the index part) or,
// when Ls is given, from a key's support array.
template <int M>
__device__ void support_columns(const uint64_t *buf, const uint16_t *Ls, const uint32_t *gb, uint32_t *mat,
                                const KgDims &d, int grp)
{
    const int n = d.n, t = d.t;
    uint32_t Lb[M];
#pragma unroll
    for (int k = 0; k < M; k++)
        Lb[k] = 0;
    uint32_t valid = 0;
    for (int c = 0; c < 32; c++) {
        const int i = 32 * grp + c;
        if (i < n) {
            const uint32_t L = Ls ? (uint32_t)Ls[i] : bitrev_m((uint32_t)(buf[i] & (uint64_t)(d.q - 1)), M);
            valid |= 1u << c;
#pragma unroll
            for (int k = 0; k < M; k++)
                Lb[k] |= ((L >> k) & 1u) << c;
        }
    }
    uint32_t e[M], v[M];
#pragma unroll
    for (int k = 0; k < M; k++)
        e[k] = gb[t * 13 + k];
    for (int j = t - 1; j >= 0; j--) {
        bs_mul<M>(e, e, Lb);
#pragma unroll
        for (int k = 0; k < M; k++)
            e[k] ^= gb[j * 13 + k];
    }
    bs_inv<M>(v, e);  // g has no roots in GF(2^m): e is never 0 on a valid column
    for (int j = 0; j < t; j++) {
#pragma unroll
        for (int k = 0; k < M; k++)
            mat[(size_t)(j * M + k) * d.rw + grp] = v[k] & valid;
        bs_mul<M>(v, v, Lb);
    }
}

__global__ void __launch_bounds__(SUP_THREADS) k_kg_support(uint8_t *__restrict__ work, KgDims d)
{
    extern __shared__ __align__(16) uint8_t sm_sup[];
    uint64_t *buf = reinterpret_cast<uint64_t *>(sm_sup);
    uint32_t *gb = reinterpret_cast<uint32_t *>(buf + d.q);  // [t + 1][13]: g_j as bitsliced constants
    __shared__ int s_dup;
    uint8_t *wk = work + (size_t)blockIdx.x * d.stride;
    PanelInfo *pinfo = reinterpret_cast<PanelInfo *>(wk + d.off_panel);
    if (pinfo->status != KG_OK)
        return;
    const int tid = threadIdx.x, q = d.q, q1 = q - 1, t = d.t, m = d.m, n = d.n;
    const uint8_t *pm = wk + d.off_r + d.n / 8;  // the 2^m random words
    for (int i = tid; i < q; i += SUP_THREADS) {
        const uint32_t w = pm[4 * i] | (pm[4 * i + 1] << 8) | (pm[4 * i + 2] << 16) | ((uint32_t)pm[4 * i + 3] << 24);
        buf[i] = ((uint64_t)w << 31) | (uint64_t)i;
    }
    const uint16_t *irr = reinterpret_cast<const uint16_t *>(wk + d.off_irr);
    for (int e = tid; e < (t + 1) * 13; e += SUP_THREADS) {
        const int j = e / 13, k = e - j * 13;
        const uint32_t gj = j < t ? irr[j] : 1u;
        gb[e] = 0u - ((gj >> k) & 1u);
    }
    if (tid == 0)
        s_dup = 0;
    seg_sort(buf, q, m);
    for (int i = 1 + tid; i < q; i += SUP_THREADS)
        if ((buf[i - 1] >> 31) == (buf[i] >> 31))
            s_dup = 1;
    __syncthreads();
    if (s_dup) {
        if (tid == 0)
            pinfo->status = KG_PERM;
        return;
    }
    int16_t *pi = reinterpret_cast<int16_t *>(wk + d.off_pi);
    for (int i = tid; i < q; i += SUP_THREADS)
        pi[i] = (int16_t)(buf[i] & (uint64_t)q1);
    // one thread per 32-column group
    uint32_t *mat = reinterpret_cast<uint32_t *>(wk + d.off_mat);
    const int groups = (n + 31) / 32;
    for (int grp = tid; grp < groups; grp += SUP_THREADS) {
        if (m == 12)
            support_columns<12>(buf, nullptr, gb, mat, d, grp);
        else
            support_columns<13>(buf, nullptr, gb, mat, d, grp);
    }
    for (int e = tid; e < d.mt * (d.rw - groups); e += SUP_THREADS) {
        const int r = e / (d.rw - groups), w = groups + e % (d.rw - groups);
        mat[(size_t)r * d.rw + w] = 0;
    }
}

// The parity-check matrix of an existing key (its support L, n entries, and
// Goppa polynomial g, t + 1 coefficients with g[t] = 1, as the key expansion
// keeps them on the device) into workspace slot 0, for the elimination that
// gives the key's public key (pk_gen.c:52-113 from a stored key).
__global__ void __launch_bounds__(SUP_THREADS) k_kg_support_key(uint8_t *__restrict__ work, KgDims d,
                                                                const uint16_t *__restrict__ L,
                                                                const uint16_t *__restrict__ g)
{
    __shared__ uint32_t gb[(128 + 1) * 13];  // g_j as bitsliced constants
    const int tid = threadIdx.x, t = d.t, n = d.n;
    PanelInfo *pinfo = reinterpret_cast<PanelInfo *>(work + d.off_panel);
    for (int e = tid; e < (t + 1) * 13; e += SUP_THREADS) {
        const int j = e / 13, k = e - j * 13;
        gb[e] = 0u - (((uint32_t)g[j] >> k) & 1u);
    }
    if (tid == 0)
        pinfo->status = KG_OK;
    __syncthreads();
    uint32_t *mat = reinterpret_cast<uint32_t *>(work + d.off_mat);
    const int groups = (n + 31) / 32;
    for (int grp = tid; grp < groups; grp += SUP_THREADS) {
        if (d.m == 12)
            support_columns<12>(nullptr, L, gb, mat, d, grp);
        else
            support_columns<13>(nullptr, L, gb, mat, d, grp);
    }
    for (int e = tid; e < d.mt * (d.rw - groups); e += SUP_THREADS) {
        const int r = e / (d.rw - groups), w = groups + e % (d.rw - groups);
        mat[(size_t)r * d.rw + w] = 0;
    }
}

// ---- 4. elimination ---------------------------------------------------------
constexpr int PANEL_THREADS = 256;

// Pivot rows of panel p (columns 32p .. 32p + npiv - 1).  Warp 0 walks the
// rows not yet holding a pivot, 32 at a time, and keeps a reduced basis of
// their panel words (lane b holds the vector with leading bit b and which
// chosen rows it combines); a row whose word is independent of the basis is
// chosen.  When npiv rows are chosen the basis is the identity on the panel
// columns and its combinations are the transform T.  Then the chosen rows are
// copied aside for k_ge_apply, which overwrites them.
__global__ void __launch_bounds__(PANEL_THREADS) k_ge_panel(uint8_t *__restrict__ work, KgDims d, int p)
{
    __shared__ uint32_t s_src[PANEL];
    __shared__ int s_n;
    uint8_t *wk = work + (size_t)blockIdx.x * d.stride;
    PanelInfo *pi = reinterpret_cast<PanelInfo *>(wk + d.off_panel);
    if (pi->status != KG_OK)
        return;
    const uint32_t *mat = reinterpret_cast<const uint32_t *>(wk + d.off_mat);
    uint8_t *used = wk + d.off_used;
    const int tid = threadIdx.x, lane = tid & 31, c0 = PANEL * p, npiv = min(PANEL, d.mt - c0);
    const uint32_t pmask = npiv == 32 ? 0xFFFFFFFFu : (1u << npiv) - 1u;
    if (p == 0) {
        for (int r = tid; r < d.mt; r += PANEL_THREADS)
            used[r] = 0;
        if (tid == 0)
            pi->scan0 = 0;
    }
    __syncthreads();
    if (tid < 32) {
        const unsigned F = 0xFFFFFFFFu;
        uint32_t basis = 0, btag = 0;  // this lane's basis vector (leading bit = lane)
        bool have = false;
        int nsel = 0;
        for (int base = pi->scan0; base < d.mt && nsel < npiv; base += 32) {
            const int r = base + lane;
            const uint32_t w = (r < d.mt && !used[r]) ? mat[(size_t)r * d.rw + p] & pmask : 0u;
            uint32_t cm = __ballot_sync(F, w != 0);
            while (cm && nsel < npiv) {
                const int j = __ffs(cm) - 1;
                cm &= cm - 1;
                uint32_t v = __shfl_sync(F, w, j);
                // the basis is reduced, so its vectors for v's set leading bits
                // clear exactly those bits
                const bool hit = have && ((v >> lane) & 1u);
                v ^= __reduce_xor_sync(F, hit ? basis : 0u);
                const uint32_t tg = __reduce_xor_sync(F, hit ? btag : 0u);
                if (v) {
                    const int lb = __ffs(v) - 1;
                    const uint32_t ntag = tg ^ (1u << nsel);
                    if (have && ((basis >> lb) & 1u)) {
                        basis ^= v;
                        btag ^= ntag;
                    }
                    if (lane == lb) {
                        basis = v;
                        btag = ntag;
                        have = true;
                    }
                    if (lane == 0)
                        s_src[nsel] = (uint32_t)(base + j);
                    nsel++;
                }
            }
        }
        if (lane == 0)
            s_n = nsel;
        if (nsel == npiv && lane < npiv)
            pi->T[lane] = btag;
    }
    __syncthreads();
    if (s_n < npiv) {
        if (tid == 0)
            pi->status = KG_SINGULAR;
        return;
    }
    uint32_t *prow = reinterpret_cast<uint32_t *>(wk + d.off_prow);
    if (tid < npiv) {
        pi->src[tid] = s_src[tid];
        prow[c0 + tid] = s_src[tid];
        used[s_src[tid]] = 1;
    }
    __syncthreads();
    if (tid < 32) {
        // the first row not yet used, 32 rows per ballot (rows past mt stop it)
        int z = pi->scan0;
        for (;;) {
            const int r = z + lane;
            const uint32_t free_rows = __ballot_sync(0xFFFFFFFFu, r >= d.mt || !used[r]);
            if (free_rows) {
                z += __ffs(free_rows) - 1;
                break;
            }
            z += 32;
        }
        if (lane == 0) {
            pi->npiv = npiv;
            pi->scan0 = min(z, d.mt);
        }
    }
    // copies of the chosen rows, 16-byte columns from word p & ~3 (the
    // update's layout), four loads in flight per thread
    uint4 *cp = reinterpret_cast<uint4 *>(wk + d.off_src);
    const uint4 *m4 = reinterpret_cast<const uint4 *>(mat);
    const int rw4 = d.rw / 4, q0 = p / 4, W4 = rw4 - q0, items = npiv * W4;
    for (int e0 = tid; e0 < items; e0 += 4 * PANEL_THREADS) {
        uint4 v[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = e0 + u * PANEL_THREADS;
            if (e < items) {
                const int j = e / W4, w = q0 + e % W4;
                v[u] = m4[(size_t)s_src[j] * rw4 + w];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = e0 + u * PANEL_THREADS;
            if (e < items) {
                const int j = e / W4, w = q0 + e % W4;
                cp[j * rw4 + w] = v[u];
            }
        }
    }
}

constexpr int APPLY_THREADS = 1024;
constexpr int APPLY_ROWS = 384;  // most rows per block (fewer when few attempts run: more blocks)

// Shared memory of k_ge_apply: 8 groups x 16 combinations x the active width.
size_t apply_smem(int width) { return (size_t)8 * 16 * width * 4; }

// Every row, words p4 = p & ~3 ..: a chosen row becomes its reduced pivot
// row, every other row gets its panel columns cleared.  Both are XORs of the
// copied chosen rows: row r with panel word x absorbs the reduced pivots of
// x's bits, i.e. the chosen rows selected by x' = XOR of T[b] over the bits b
// of x.  That XOR is found four bits of x' at a time in tables of all 16
// combinations of four chosen rows (the "four Russians" method), built per
// block in shared memory.  Each thread carries four consecutive words
// (16-byte loads, stores and table reads); words p4 .. p - 1 are zero in
// every chosen row.
__global__ void __launch_bounds__(APPLY_THREADS) k_ge_apply(uint8_t *__restrict__ work, KgDims d, int p, int rows)
{
    extern __shared__ __align__(16) uint4 s_tab4[];  // [8][16][W4]
    __shared__ uint32_t s_x[APPLY_ROWS];             // x' of each row
    __shared__ uint8_t s_own[APPLY_ROWS];            // 0: chosen row (its own content is replaced)
    __shared__ uint32_t s_T[PANEL], s_srcr[PANEL];
    uint8_t *wk = work + (size_t)blockIdx.x * d.stride;
    const PanelInfo *pi = reinterpret_cast<const PanelInfo *>(wk + d.off_panel);
    if (pi->status != KG_OK)
        return;
    uint32_t *mat = reinterpret_cast<uint32_t *>(wk + d.off_mat);
    const uint32_t *cp = reinterpret_cast<const uint32_t *>(wk + d.off_src);
    const int npiv = pi->npiv, p4 = p & ~3, W4 = (d.rw - p4) / 4, tid = threadIdx.x;
    const int rw4 = d.rw / 4;
    const uint32_t pmask = npiv == 32 ? 0xFFFFFFFFu : (1u << npiv) - 1u;
    const int r0 = blockIdx.y * rows, nrows = min(rows, d.mt - r0);
    if (tid < PANEL) {
        s_T[tid] = tid < npiv ? pi->T[tid] : 0u;
        s_srcr[tid] = tid < npiv ? pi->src[tid] : 0xFFFFFFFFu;
    }
    // tables: tab[g][c][w4] = XOR of chosen rows 4g + b for the bits b of c
    const uint4 *cp4 = reinterpret_cast<const uint4 *>(cp + p4);
    for (int e = tid; e < 8 * W4; e += APPLY_THREADS) {
        const int g = e / W4, w4 = e - g * W4;
        uint4 v[4];
#pragma unroll
        for (int b = 0; b < 4; b++)
            v[b] = 4 * g + b < npiv ? cp4[(4 * g + b) * rw4 + w4] : make_uint4(0, 0, 0, 0);
        uint4 *t = s_tab4 + g * 16 * W4 + w4;
#pragma unroll
        for (int c = 0; c < 16; c++) {
            uint4 x = make_uint4(0, 0, 0, 0);
#pragma unroll
            for (int b = 0; b < 4; b++)
                if (c & (1 << b)) {
                    x.x ^= v[b].x;
                    x.y ^= v[b].y;
                    x.z ^= v[b].z;
                    x.w ^= v[b].w;
                }
            t[c * W4] = x;
        }
    }
    __syncthreads();
    // each row's x' and whether it keeps its own content, read before any
    // row is written
    for (int t = tid; t < nrows; t += APPLY_THREADS) {
        const int r = r0 + t;
        int b = -1;
        for (int i = 0; i < npiv; i++)
            if ((int)s_srcr[i] == r)
                b = i;
        uint32_t x;
        if (b >= 0) {
            x = s_T[b];
        } else {
            uint32_t pw = mat[(size_t)r * d.rw + p] & pmask;
            x = 0;
            while (pw) {
                x ^= s_T[__ffs(pw) - 1];
                pw &= pw - 1;
            }
        }
        s_x[t] = x;
        s_own[t] = b < 0;
    }
    __syncthreads();
    // thread (t0, w4): 16-byte column w4 of rows t0, t0 + 16, ...
    const int w4 = tid & 63;
    if (w4 >= W4)
        return;
    uint4 *col = reinterpret_cast<uint4 *>(mat + p4) + w4;  // row r: col[r * rw4]
    const uint4 *tg = s_tab4 + w4;  // table g, combination c: tg[(16 g + c) * W4]
    constexpr int STEP = APPLY_THREADS / 64, U = 2;  // two rows in flight per thread
    for (int t = tid >> 6; t < nrows; t += U * STEP) {
        uint4 acc[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int tu = t + u * STEP;
            acc[u] = make_uint4(0, 0, 0, 0);
            if (tu < nrows && s_own[tu])
                acc[u] = col[(r0 + tu) * rw4];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int tu = t + u * STEP;
            if (tu >= nrows)
                continue;
            const uint32_t x = s_x[tu];
#pragma unroll
            for (int g = 0; g < 8; g++) {
                const uint4 v = tg[(16 * g + (int)((x >> (4 * g)) & 15u)) * W4];
                acc[u].x ^= v.x;
                acc[u].y ^= v.y;
                acc[u].z ^= v.z;
                acc[u].w ^= v.w;
            }
            col[(r0 + tu) * rw4] = acc[u];
        }
    }
}

// ---- 5. control bits ----------------------------------------------------------
constexpr int CB_THREADS = 1024;

// Six int16 arrays of 2^m entries and the bit array.
size_t cbits_smem(const KgDims &d) { return (size_t)6 * d.q * 2 + (size_t)(d.cond + 3) / 4 * 4; }

__device__ __forceinline__ uint32_t rev_bits(uint32_t s, int nb) { return nb ? __brev(s) >> (32 - nb) : 0; }

// Control bit `gb` is bit gb % 8 of byte gb / 8 (controlbits.c:17-18).
__device__ __forceinline__ void put_bit(uint32_t *bits, long gb, uint32_t v)
{
    if (v)
        atomicOr(&bits[gb >> 5], 1u << (gb & 31));
}

// All sub-networks of a recursion level at once: at level lev the 2^lev
// segments of ns = 2^(m - lev) entries each hold one inner permutation (local
// values 0..ns-1).  controlbits.c:22-170 reaches each quantity below with
// constant-time sorts; here each is the permutation inverse or composition
// that sort performs, by scatter or gather in shared memory.
__global__ void __launch_bounds__(CB_THREADS) k_kg_controlbits(uint8_t *__restrict__ work, KgDims d)
{
    extern __shared__ __align__(16) uint8_t sm_cb[];
    int16_t *Pa = reinterpret_cast<int16_t *>(sm_cb);  // current permutations
    int16_t *Ia = Pa + d.q;                             // their inverses
    int16_t *Ba = Ia + d.q;                             // pibar, later M
    int16_t *Ca = Ba + d.q;                             // cycle labels c
    int16_t *Qa = Ca + d.q;                             // pibar^(2^k)
    int16_t *Ta = Qa + d.q;                             // F(pi(x))
    uint32_t *bits = reinterpret_cast<uint32_t *>(Ta + d.q);
    __shared__ int s_bad;
    uint8_t *wk = work + (size_t)blockIdx.x * d.stride;
    PanelInfo *pinfo = reinterpret_cast<PanelInfo *>(wk + d.off_panel);
    if (pinfo->status != KG_OK)
        return;
    const int tid = threadIdx.x, m = d.m, n = d.q, half = n / 2;
    const int16_t *pig = reinterpret_cast<const int16_t *>(wk + d.off_pi);
    for (int i = tid; i < (d.cond + 3) / 4; i += CB_THREADS)
        bits[i] = 0;
    for (int x = tid; x < n; x += CB_THREADS)
        Pa[x] = pig[x];
    if (tid == 0)
        s_bad = 0;
    __syncthreads();
    for (int lev = 0; lev < m - 1; lev++) {
        const int w = m - lev, ns = n >> lev, h = ns / 2;
        // inverse
        for (int x = tid; x < n; x += CB_THREADS) {
            const int lx = x & (ns - 1), base = x - lx;
            Ia[base + Pa[x]] = (int16_t)lx;
        }
        __syncthreads();
        // pibar(y) = pi(pi^-1(y ^ 1) ^ 1)
        for (int x = tid; x < n; x += CB_THREADS) {
            const int lx = x & (ns - 1), base = x - lx;
            Ba[x] = Pa[base + (Ia[base + (lx ^ 1)] ^ 1)];
        }
        __syncthreads();
        // c = min(x, pibar(x)); Q = pibar^2
        for (int x = tid; x < n; x += CB_THREADS) {
            const int lx = x & (ns - 1), base = x - lx, pb = Ba[x];
            Ca[x] = (int16_t)min(lx, pb);
            Qa[x] = Ba[base + pb];
        }
        __syncthreads();
        // w - 2 times: c <- min(c, c o Q), Q <- Q o Q
        for (int it = 1; it < w - 1; it++) {
            int cn[KG_MAX_Q / CB_THREADS], qn[KG_MAX_Q / CB_THREADS];
#pragma unroll
            for (int e = 0; e < KG_MAX_Q / CB_THREADS; e++) {
                const int x = tid + CB_THREADS * e;
                if (x < n) {
                    const int lx = x & (ns - 1), base = x - lx, qx = base + Qa[x];
                    cn[e] = min((int)Ca[x], (int)Ca[qx]);
                    qn[e] = Qa[qx];
                }
            }
            __syncthreads();
#pragma unroll
            for (int e = 0; e < KG_MAX_Q / CB_THREADS; e++) {
                const int x = tid + CB_THREADS * e;
                if (x < n) {
                    Ca[x] = (int16_t)cn[e];
                    Qa[x] = (int16_t)qn[e];
                }
            }
            __syncthreads();
        }
        // first layer: pair j swaps when c(2j) is odd (F); T = F o pi
        for (int x = tid; x < n; x += CB_THREADS) {
            const int lx = x & (ns - 1), base = x - lx, s = x / ns;
            if (!(lx & 1))
                put_bit(bits, (long)lev * half + rev_bits(s, lev) + (long)(lx >> 1) * (1 << lev), Ca[x] & 1);
            const int px = Pa[x];
            Ta[x] = (int16_t)(px ^ (Ca[base + (px & ~1)] & 1));
        }
        __syncthreads();
        // last layer: pair k swaps when T(2k) is odd (L); M(L(x)) = T(x)
        for (int x = tid; x < n; x += CB_THREADS) {
            const int lx = x & (ns - 1), base = x - lx, s = x / ns;
            const int l = Ta[base + (lx & ~1)] & 1;
            if (!(lx & 1))
                put_bit(bits, (long)lev * half + rev_bits(s, lev) + (long)(2 * w - 2) * half + (long)(lx >> 1) * (1 << lev),
                        l);
            Ba[base + (lx ^ l)] = Ta[x];
        }
        __syncthreads();
        // the two inner problems: M(2j)/2 in the first half, M(2j+1)/2 in the second
        for (int x = tid; x < n; x += CB_THREADS) {
            const int lx = x & (ns - 1), base = x - lx;
            const int src = lx < h ? base + 2 * lx : base + 2 * (lx - h) + 1;
            Pa[x] = (int16_t)(Ba[src] >> 1);
        }
        __syncthreads();
    }
    // w = 1: the pair swaps when pi(0) = 1
    for (int x = 2 * tid; x < n; x += 2 * CB_THREADS)
        put_bit(bits, (long)(m - 1) * half + rev_bits(x >> 1, m - 1), Pa[x] & 1);
    __syncthreads();
    // check: layers 0..m-1 then m-2..0 (stride 2^s) applied to the identity
    // must give pi (controlbits.c:193-212)
    int16_t *X = Ia;
    for (int i = tid; i < n; i += CB_THREADS)
        X[i] = (int16_t)i;
    for (int layer = 0; layer < 2 * m - 1; layer++) {
        const int sh = layer < m ? layer : 2 * m - 2 - layer;
        __syncthreads();
        for (int k = tid; k < half; k += CB_THREADS) {
            const long gb = (long)layer * half + k;
            const int blk = k >> sh, j = k & ((1 << sh) - 1);
            const int a = blk * (2 << sh) + j, b = a + (1 << sh);
            if ((bits[gb >> 5] >> (gb & 31)) & 1u) {
                const int16_t u = X[a];
                X[a] = X[b];
                X[b] = u;
            }
        }
    }
    __syncthreads();
    for (int i = tid; i < n; i += CB_THREADS)
        if (X[i] != pig[i])
            s_bad = 1;
    __syncthreads();
    uint8_t *cond = wk + d.off_cond;
    const uint8_t *bb = reinterpret_cast<const uint8_t *>(bits);
    for (int i = tid; i < d.cond; i += CB_THREADS)
        cond[i] = bb[i];
    if (tid == 0 && s_bad)
        pinfo->status = KG_CBITS;
}

// ---- 6. outputs ---------------------------------------------------------------
// For each accepted slot of the list: sk = seed | 0xFFFFFFFF as 8 little-endian
// bytes | g (2t) | control bits | s (operations.c:60-100) and pk row r =
// bytes mt/8 .. of the reduced row holding pivot r, into output position i
// of the list.
__global__ void k_kg_output(const uint8_t *__restrict__ work, const uint8_t *__restrict__ slot_seed,
                            const int *__restrict__ slots, uint8_t *__restrict__ pk, uint8_t *__restrict__ sk, KgDims d)
{
    const int i = blockIdx.x, slot = slots[i];
    const uint8_t *wk = work + (size_t)slot * d.stride;
    uint8_t *skp = sk + (size_t)i * d.sk;
    const int off_irr = 40, off_cond = 40 + 2 * d.t, off_s = off_cond + d.cond;
    for (int x = blockIdx.y * blockDim.x + threadIdx.x; x < d.sk; x += gridDim.y * blockDim.x) {
        uint8_t v;
        if (x < 32)
            v = slot_seed[(size_t)slot * 32 + x];
        else if (x < 40)
            v = x < 36 ? 0xFF : 0;
        else if (x < off_cond)
            v = wk[d.off_irr + (x - off_irr)];
        else if (x < off_s)
            v = wk[d.off_cond + (x - off_cond)];
        else
            v = wk[d.off_r + (x - off_s)];
        skp[x] = v;
    }
    const uint8_t *mat = wk + d.off_mat;
    const uint32_t *prow = reinterpret_cast<const uint32_t *>(wk + d.off_prow);
    uint8_t *pkp = pk + (size_t)i * d.mt * d.pk_row;
    const size_t total = (size_t)d.mt * d.pk_row;
    for (size_t e = (size_t)blockIdx.y * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.y * blockDim.x) {
        const int r = (int)(e / d.pk_row), b = (int)(e % d.pk_row);
        pkp[e] = mat[(size_t)prow[r] * d.rw * 4 + d.mt / 8 + b];
    }
}

// Status and next seed of every key of the round, packed for one copy.
__global__ void k_kg_collect(const uint8_t *__restrict__ work, KgDims d, int K, uint8_t *__restrict__ out)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < K * 9; e += gridDim.x * blockDim.x) {
        const int k = e / 9, w = e % 9;
        const uint8_t *wk = work + (size_t)k * d.stride;
        uint32_t v;
        if (w == 0) {
            v = (uint32_t)reinterpret_cast<const PanelInfo *>(wk + d.off_panel)->status;
        } else {
            const uint8_t *sd = wk + d.off_r + d.rlen - 32 + 4 * (w - 1);
            v = sd[0] | (sd[1] << 8) | (sd[2] << 16) | ((uint32_t)sd[3] << 24);
        }
        reinterpret_cast<uint32_t *>(out)[e] = v;
    }
}

// T's columns from the reduced matrix of slot 0: column c (< n - mt) is bit
// mt + c of the reduced pivot rows 0 .. mt - 1, word w of it (rows 32w ..
// 32w + 31) at cols[c * cwp + w]; words from the last row on are zero.  Warp
// (chunk, w): lane b takes 32 bits of pivot row 32w + b from column mt +
// 32 chunk on, and 32 ballots turn the 32 x 32 block around.
__global__ void __launch_bounds__(256) k_kg_pk_columns(const uint8_t *__restrict__ work, KgDims d,
                                                      uint32_t *__restrict__ cols, int cwp)
{
    const PanelInfo *pinfo = reinterpret_cast<const PanelInfo *>(work + d.off_panel);
    const int xc = d.n - d.mt, chunks = (xc + 31) / 32;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (pinfo->status != KG_OK || warp >= chunks * cwp)
        return;
    const int chunk = warp / cwp, w = warp - chunk * cwp, r = 32 * w + lane;
    const uint32_t *mat = reinterpret_cast<const uint32_t *>(work + d.off_mat);
    const uint32_t *prow = reinterpret_cast<const uint32_t *>(work + d.off_prow);
    uint32_t bits = 0;
    if (r < d.mt) {
        const uint32_t *row = mat + (size_t)prow[r] * d.rw;
        const int b0 = d.mt + 32 * chunk, w0 = b0 >> 5, sh = b0 & 31;
        const uint32_t lo = row[w0], hi = w0 + 1 < d.rw ? row[w0 + 1] : 0u;
        bits = __funnelshift_r(lo, hi, sh);
    }
    uint32_t mine = 0;
#pragma unroll
    for (int k = 0; k < 32; k++) {
        const uint32_t bal = __ballot_sync(0xFFFFFFFFu, (bits >> k) & 1u);
        if (lane == k)
            mine = bal;
    }
    const int c = 32 * chunk + lane;
    if (c < xc)
        cols[(size_t)c * cwp + w] = mine;
}

int set_smem_attr(const void *fn, size_t bytes)
{
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "keygen smem attribute");
}

}  // namespace

int kg_pubkey_columns(cmd_engine *eng, int set, const uint16_t *d_L, const uint16_t *d_g, uint32_t *d_cols, int cwp)
{
    std::lock_guard<std::mutex> lk(eng->mu);
    cudaSetDevice(eng->device);
    const KgDims d = kg_dims(set);
    int rc = eng->keygen.reserve(eng, d.stride);
    if (rc)
        return rc;
    uint8_t *work = static_cast<uint8_t *>(eng->keygen.ptr);
    if ((rc = set_smem_attr((const void *)k_ge_apply, apply_smem(d.rw))))
        return rc;
    cudaStream_t s = eng->stream;
    LaunchCounter lc{&eng->launches};
    k_kg_support_key<<<1, SUP_THREADS, 0, s>>>(work, d, d_L, d_g);
    const int npanels = (d.mt + PANEL - 1) / PANEL;
    // one key: small row blocks, about two per SM
    const int rows = std::min(APPLY_ROWS, std::max(32, ((d.mt + 2 * eng->num_sms - 1) / (2 * eng->num_sms) + 15) / 16 * 16));
    const int gy = (d.mt + rows - 1) / rows;
    for (int p = 0; p < npanels; p++) {
        k_ge_panel<<<1, PANEL_THREADS, 0, s>>>(work, d, p);
        k_ge_apply<<<dim3(1, gy), APPLY_THREADS, apply_smem(d.rw - (p & ~3)), s>>>(work, d, p, rows);
    }
    const int warps = (d.n - d.mt + 31) / 32 * cwp;
    k_kg_pk_columns<<<(warps + 7) / 8, 256, 0, s>>>(work, d, d_cols, cwp);
    lc.bump(2 + 2 * (uint64_t)npanels);
    int status = KG_SINGULAR;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&status, work + d.off_panel, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return cuda_fail(e, "public key derivation");
    if (status != KG_OK) {
        set_last_error("the secret key's public key has no systematic form");
        return CMD_E_ARG;
    }
    return CMD_OK;
}

}  // namespace cmd

using namespace cmd;

extern "C" {

int cmd_kem_keypair_batch(cmd_engine *eng, cmd_set set, const uint8_t *h_seeds, size_t count, uint8_t *h_pk,
                          uint8_t *h_sk, uint32_t *h_attempts, uint32_t max_attempts)
{
    if (!eng || !valid_set(set) || !h_seeds || !h_pk || !h_sk || count == 0 || count > 4096)
        return CMD_E_ARG;
    if (max_attempts == 0)
        max_attempts = 1000;
    std::lock_guard<std::mutex> lk(eng->mu);
    cudaSetDevice(eng->device);
    const KgDims d = kg_dims(set);
    const size_t pk_bytes = (size_t)d.mt * d.pk_row;
    // Attempt slots per round: about two support CTAs per SM; up to SPEC
    // attempts of one key run side by side (the reference's retries of a key
    // form a fixed chain of seeds, so later attempts can start before earlier
    // ones are decided; the first accepted one is kept).  Each pending key
    // keeps its next SPEC expansions in a chain, refilled on a second stream
    // while the round's other stages run.
    size_t cap = (size_t)std::max(32, 2 * eng->num_sms);
    // chain entry: expansion | g (2t bytes) | status
    const size_t r_stride = (d.rlen + 255) / 256 * 256 + 512;
    const size_t chain_bytes = count * SPEC * (r_stride + 32) + count * (32 + 4);
    const size_t fixed = 2048 + chain_bytes;
    // per slot: workspace, seed, collect record, list entry, one pk and sk
    auto need = [&](size_t c) { return fixed + c * (d.stride + 32 + 36 + 4 + pk_bytes + d.sk); };
    while (cap > 1 && eng->keygen.reserve(eng, need(cap)) != CMD_OK)
        cap /= 2;
    if (cap == 1 && eng->keygen.reserve(eng, need(1)) != CMD_OK)
        return CMD_E_BUDGET;
    uint8_t *mem = static_cast<uint8_t *>(eng->keygen.ptr);
    uint8_t *d_work = mem;
    uint8_t *d_chain = d_work + cap * d.stride;                 // count x SPEC x r_stride
    uint8_t *d_chain_seed = d_chain + count * SPEC * r_stride;  // count x SPEC x 32
    uint8_t *d_seeds = d_chain_seed + count * SPEC * 32;        // count x 32
    int *d_keys = reinterpret_cast<int *>(d_seeds + count * 32);  // count
    uint8_t *d_slot_seed = reinterpret_cast<uint8_t *>(d_keys + count);
    uint32_t *d_col = reinterpret_cast<uint32_t *>(d_slot_seed + cap * 32);  // 9 words a slot
    int *d_list = reinterpret_cast<int *>(d_col + cap * 9);
    uint8_t *d_pk = reinterpret_cast<uint8_t *>(d_list + cap);
    uint8_t *d_sk = d_pk + cap * pk_bytes;
    cudaStream_t s = eng->stream;
    LaunchCounter lc{&eng->launches};
    int rc = CMD_OK;
    const size_t smem_gp = genpoly_smem(d), smem_sup = support_smem(d), smem_cb = cbits_smem(d);
    const size_t smem_apply = apply_smem(d.rw);
    if ((rc = set_smem_attr((const void *)k_kg_genpoly, smem_gp)) || (rc = set_smem_attr((const void *)k_kg_support, smem_sup)) ||
        (rc = set_smem_attr((const void *)k_kg_controlbits, smem_cb)) ||
        (rc = set_smem_attr((const void *)k_ge_apply, smem_apply)))
        return rc;
    // s2: the next chains (expansion, Goppa polynomial); s3: the copies of
    // finished key pairs to the host, overlapping the next round on s
    cudaStream_t s2 = nullptr, s3 = nullptr;
    cudaEvent_t ev_fill = nullptr, ev_exp = nullptr, ev_out = nullptr, ev_copied = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s3, cudaStreamNonBlocking);
    for (cudaEvent_t *ev : {&ev_fill, &ev_exp, &ev_out, &ev_copied})
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    // every key's first chain, from its seed
    std::vector<int> keys(count);
    for (size_t i = 0; i < count; i++)
        keys[i] = (int)i;
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_seeds, h_seeds, count * 32, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_keys, keys.data(), count * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_kg_expand<<<(int)count, 32, 0, s>>>(d_seeds, d_keys, d_chain, d_chain_seed, d, (int)count, 0, r_stride);
        k_kg_genpoly<<<(int)(count * SPEC), GP_THREADS, smem_gp, s>>>(d_chain, d_keys, d, r_stride);
        lc.bump(2);
        e = cudaEventRecord(ev_exp, s);
    }
    // keys still to finish, by output index
    std::vector<int> pend(count);
    std::vector<uint32_t> tries(count, 0);
    for (size_t i = 0; i < count; i++)
        pend[i] = (int)i;
    std::vector<uint32_t> col;
    std::vector<int> list, list_out;
    while (!pend.empty() && e == cudaSuccess && rc == CMD_OK) {
        std::vector<int> still;
        const size_t keys_per_chunk = std::min(pend.size(), cap);
        const int D = (int)std::max<size_t>(1, std::min<size_t>(SPEC, cap / keys_per_chunk));
        for (size_t base = 0; base < pend.size() && e == cudaSuccess && rc == CMD_OK; base += keys_per_chunk) {
            const int K = (int)std::min(keys_per_chunk, pend.size() - base), S = K * D;
            // the chains this chunk reads are complete (every expansion so far
            // is on s2 before ev_exp); the key list goes to a free region
            int *kd = d_keys + base;
            if ((e = cudaStreamWaitEvent(s, ev_exp, 0)) != cudaSuccess ||
                (e = cudaMemcpyAsync(kd, pend.data() + base, (size_t)K * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess)
                break;
            k_kg_fill<<<S, 256, 0, s>>>(d_chain, d_chain_seed, kd, d_work, d_slot_seed, d, D, r_stride);
            // next chains of these keys (attempts D .. D + SPEC - 1 from now),
            // overlapping the stages below
            if ((e = cudaEventRecord(ev_fill, s)) != cudaSuccess || (e = cudaStreamWaitEvent(s2, ev_fill, 0)) != cudaSuccess)
                break;
            k_kg_expand<<<K, 32, 0, s2>>>(nullptr, kd, d_chain, d_chain_seed, d, K, D, r_stride);
            k_kg_genpoly<<<K * SPEC, GP_THREADS, smem_gp, s2>>>(d_chain, kd, d, r_stride);
            if ((e = cudaEventRecord(ev_exp, s2)) != cudaSuccess)
                break;
            lc.bump(3);
            k_kg_support<<<S, SUP_THREADS, smem_sup, s>>>(d_work, d);
            const int npanels = (d.mt + PANEL - 1) / PANEL;
            // rows per update block: about two blocks per SM over the round's slots
            const int per_slot = std::max(1, (2 * eng->num_sms + S - 1) / S);
            const int rows = std::min(APPLY_ROWS, std::max(32, ((d.mt + per_slot - 1) / per_slot + 15) / 16 * 16));
            const int gy = (d.mt + rows - 1) / rows;
            for (int p = 0; p < npanels; p++) {
                k_ge_panel<<<S, PANEL_THREADS, 0, s>>>(d_work, d, p);
                k_ge_apply<<<dim3(S, gy), APPLY_THREADS, apply_smem(d.rw - (p & ~3)), s>>>(d_work, d, p, rows);
            }
            k_kg_controlbits<<<S, CB_THREADS, smem_cb, s>>>(d_work, d);
            k_kg_collect<<<(S * 9 + 255) / 256, 256, 0, s>>>(d_work, d, S, reinterpret_cast<uint8_t *>(d_col));
            lc.bump(3 + 2 * (uint64_t)npanels);
            col.resize((size_t)S * 9);
            if ((e = cudaGetLastError()) != cudaSuccess ||
                (e = cudaMemcpyAsync(col.data(), d_col, (size_t)S * 36, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess)
                break;
            // per key: the first attempt that is accepted (or fails its
            // self-check) ends it; otherwise it continues after its last slot
            list.clear();
            list_out.clear();
            for (int k = 0; k < K; k++) {
                const int out = pend[base + k];
                int j = 0;
                while (j < D && (int)col[(size_t)(k * D + j) * 9] != KG_OK && (int)col[(size_t)(k * D + j) * 9] != KG_CBITS)
                    j++;
                if (j == D) {
                    tries[out] += D;
                    if (tries[out] < max_attempts) {
                        still.push_back(out);
                    } else {
                        rc = CMD_E_KEYGEN;
                        set_last_error("key generation: attempt limit reached");
                    }
                    continue;
                }
                tries[out] += j + 1;
                if ((int)col[(size_t)(k * D + j) * 9] == KG_CBITS) {
                    rc = CMD_E_KEYGEN;
                    set_last_error("key generation: control bits do not reproduce the permutation");
                    continue;
                }
                list.push_back(k * D + j);
                list_out.push_back(out);
            }
            if (list.empty())
                continue;
            const int nl = (int)list.size();
            // the previous round's key pairs have left d_pk / d_sk (a wait on
            // an event not yet recorded passes)
            if ((e = cudaMemcpyAsync(d_list, list.data(), (size_t)nl * 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(s, ev_copied, 0)) != cudaSuccess)
                break;
            k_kg_output<<<dim3(nl, 16), 256, 0, s>>>(d_work, d_slot_seed, d_list, d_pk, d_sk, d);
            lc.bump();
            if ((e = cudaEventRecord(ev_out, s)) != cudaSuccess || (e = cudaStreamWaitEvent(s3, ev_out, 0)) != cudaSuccess)
                break;
            for (int i = 0; i < nl && e == cudaSuccess; i++) {
                const int out = list_out[i];
                if ((e = cudaMemcpyAsync(h_pk + (size_t)out * pk_bytes, d_pk + (size_t)i * pk_bytes, pk_bytes,
                                         cudaMemcpyDeviceToHost, s3)) == cudaSuccess)
                    e = cudaMemcpyAsync(h_sk + (size_t)out * d.sk, d_sk + (size_t)i * d.sk, d.sk, cudaMemcpyDeviceToHost, s3);
            }
            if (e == cudaSuccess)
                e = cudaEventRecord(ev_copied, s3);
        }
        pend.swap(still);
    }
    if (h_attempts)
        for (size_t i = 0; i < count; i++)
            h_attempts[i] = tries[i];
    // the last speculative chains may still run on s2, the last copies on s3
    for (cudaStream_t st : {s3, s2}) {
        const cudaError_t e2 = st ? cudaStreamSynchronize(st) : cudaSuccess;
        if (e == cudaSuccess)
            e = e2;
    }
    for (cudaEvent_t ev : {ev_fill, ev_exp, ev_out, ev_copied})
        if (ev)
            cudaEventDestroy(ev);
    for (cudaStream_t st : {s2, s3})
        if (st)
            cudaStreamDestroy(st);
    if (e != cudaSuccess)
        return cuda_fail(e, "key generation");
    return rc;
}

int cmd_kem_keypair(cmd_engine *eng, cmd_set set, const uint8_t *h_seed, uint8_t *h_pk, uint8_t *h_sk,
                    uint32_t *attempts)
{
    return cmd_kem_keypair_batch(eng, set, h_seed, 1, h_pk, h_sk, attempts, 0);
}

}  // extern "C"
