// Engine-internal declarations shared by the CUDA launchers and the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>

#include "cmd_b200.h"
#include "params.h"

namespace cmd {

// Device-resident expanded key: one allocation carved into these arrays.
struct KeyDev {
    int set = 0;
    uint16_t *L = nullptr;      // support, n entries (support_gen output)
    uint16_t *g = nullptr;      // Goppa polynomial, t+1 coefficients, g[t] = 1
    uint16_t *ginv2 = nullptr;  // 1/g(L_i)^2 for i < n (0 where g(L_i) = 0)
    uint32_t *tab = nullptr;    // syndrome table, sb rows of twp (t rounded up to
                                // 4) words; word w < t of row b packs
                                // L_b^{2w}/g^2 (low) and L_b^{2w+1}/g^2 (high):
                                // util.c:86-100 values, rows 16-byte aligned
    uint32_t *tabd = nullptr;   // the same table, dense: sb rows of twd words,
                                // bit j*m + k of row b = bit k of L_b^j/g^2
                                // (the fused kernel's syndrome source)
    uint32_t *Lbs = nullptr;    // bitsliced support, plane-major [m][nw]:
                                // bit p of Lbs[k*nw+w] = bit k of L[32w+p]
    uint32_t *bctl = nullptr;   // Benes network as swap masks, [2m-1][2^(m-5)]:
                                // bit b of bctl[l*2^(m-5)+w] set when layer l
                                // exchanges position 32w+b (the pair's lower
                                // element) with its partner
    uint32_t *wfft = nullptr;   // 1/g(a)^2 at every field element a in the
                                // additive FFT's position order, bitsliced
                                // plane-major [m][2^(m-5)]: bit b of word w is
                                // the element a = bitrev_m(32w + b)
    uint8_t *sk = nullptr;      // device copy of the secret key bytes
};

// Records a launch against an engine counter (count of our kernels).
struct LaunchCounter {
    std::atomic<uint64_t> *ctr;
    void bump(uint64_t n = 1) const
    {
        if (ctr)
            ctr->fetch_add(n, std::memory_order_relaxed);
    }
};

cudaError_t launch_key_expand(const KeyDev &k, cudaStream_t s, LaunchCounter lc);
// Words of KeyDev::bctl for one set.
inline size_t benes_mask_words(const SetInfo &si) { return (size_t)(2 * si.m - 1) << (si.m - 5); }
// Words of KeyDev::wfft for one set.
inline size_t fft_weight_words(const SetInfo &si) { return (size_t)si.m << (si.m - 5); }

cudaError_t launch_synd_plain(const KeyDev &k, const uint8_t *d_cts, size_t count,
                              uint32_t *d_synd, cudaStream_t s, LaunchCounter lc);
cudaError_t launch_bm_plain(int set, const uint16_t *d_synd, size_t count, uint16_t *d_loc,
                            cudaStream_t s, LaunchCounter lc);
cudaError_t launch_root_plain(const KeyDev &k, const uint16_t *d_loc, size_t count,
                              uint32_t *d_err, uint16_t *d_weight, cudaStream_t s,
                              LaunchCounter lc, int num_sms);
cudaError_t launch_root_images(const KeyDev &k, const uint16_t *d_loc, size_t count,
                               uint16_t *d_images, cudaStream_t s, LaunchCounter lc);
cudaError_t preload_plain_kernels();

// Fused path: one work item = up to 32 ciphertexts of one key.
struct FusedTile {
    uint32_t key;     // index into the key table
    uint32_t count;   // 1..32
    uint64_t first;   // index of the first ciphertext of the tile in the
                      // ciphertext index list (mixed) or the batch (single)
};
struct FusedKeyRef {
    int32_t set;
    int32_t pad;
    const uint32_t *tab;
    const uint32_t *Lbs;
    const uint32_t *bctl;
};

// Additive-FFT evaluation plan of one parameter set (fft_plan.cpp): constant
// tables shared by every key of the set.
//   scalpow[d*256 + i]: b_d^i, the radix-conversion scale of depth d;
//   tw[(off_d + u)*16 + k]: plane k of twiddle word u of depth d (off_d =
//   sum of the word counts 2^(m-e-6) of the depths e < d).
struct FftPlanDev {
    const uint16_t *scalpow;
    const uint32_t *tw;
};
struct FusedArgs {
    const FusedTile *tiles;        // device list of rounds; null = implicit
                                   // rounds over one key: round r covers
                                   // ciphertexts [r*round_cts, +round_cts)
    uint32_t ntiles;               // number of rounds
    uint32_t round_cts;            // implicit mode: ciphertexts per round
    uint64_t total;                // implicit mode: batch size
    const FusedKeyRef *keys;       // device key table (null in implicit mode)
    FusedKeyRef key0;              // implicit mode: the one key
    const uint8_t *cts;            // ciphertext base pointer
    const uint64_t *ct_off;        // per-ciphertext byte offsets, or null
    const uint64_t *err_off;       // per-ciphertext error-row word offsets, or null
    const uint32_t *order;         // ciphertext index per round slot, or null
    uint32_t *err;
    uint16_t *weight;
    uint32_t *tile_counter;        // zeroed before the launch
    int single_set;                // >= 0: every round has this set
    uint32_t err_stride;           // words per error row when err_off is null
    uint16_t *pos;                 // or null: per ciphertext t+1 u16, the weight
                                   // then the error positions ascending, 0xFFFF after
    uint32_t pos_stride;           // u16 per positions row
    uint8_t *err_packed;           // or null: error rows of n/8 bytes back to back
                                   // (a host-mapped buffer), row c at c * n/8
    FftPlanDev fft[NSETS];         // root-search plans, indexed by set
};
cudaError_t launch_fused(const FusedArgs &a, int grid, int warps_per_block, cudaStream_t s,
                         LaunchCounter lc);

// Latency path (serving loop; latency.cu): one work item per ciphertext.
struct LatItem {
    const uint32_t *wfft; // key's syndrome weights in FFT order (KeyDev::wfft)
    const uint32_t *bctl; // key's support-network swap masks
    uint32_t ct_off;      // byte offset of the ciphertext in the batch
    uint32_t err_off;     // word offset of the error row in the batch
    int32_t set;
    int32_t pad;
    uint8_t *row;         // or the packed n/8-byte error row, stored here (GPU-mapped host memory)
};
// Tile path: ntiles tiles of 32 item slots (LatItem.pad = tile count, padding
// slots set -1).  d_scratch holds ntiles * TILE_SCRATCH_WORDS words: each
// tile's radix-converted locators (bitsliced, 16 words per entry), then the
// transposed-FFT sums of its ciphertexts (2^D' u16 entries x 32 slots).
constexpr int TILE_LOC_WORDS = 256 * 16;
constexpr int TILE_SUM_WORDS = 256 * 32 / 2;
constexpr int TILE_SCRATCH_WORDS = TILE_LOC_WORDS + TILE_SUM_WORDS;
struct FftPlans {
    FftPlanDev p[NSETS];
};
cudaError_t launch_tile_path(const void *d_items, const uint8_t *d_cts, uint32_t ntiles, uint32_t *d_scratch,
                             uint32_t *d_err, uint16_t *d_weight, const FftPlans &plans, cudaStream_t s,
                             LaunchCounter lc);
// The tile path over one key's batch (ciphertexts at the set's ct stride,
// error rows at its nw stride); with d_synd, only the syndromes (rows of 2t
// u16).  d_scratch: tile_single_scratch_words(count) words.
cudaError_t launch_tile_single(const KeyDev &k, const uint8_t *d_cts, size_t count, uint32_t *d_scratch,
                               uint32_t *d_err, uint16_t *d_weight, uint16_t *d_synd, const FftPlans &plans,
                               cudaStream_t s, LaunchCounter lc);
size_t tile_single_scratch_words(size_t count);

void set_last_error(const std::string &msg);

}  // namespace cmd
