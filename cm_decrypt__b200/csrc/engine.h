// Engine and key objects behind the opaque C handles, plus the helpers the
// batch, tuning and serving code share.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"

struct cmd_engine;

namespace cmd {

// Growable device buffer charged against the engine's HBM budget.
struct Scratch {
    void *ptr = nullptr;
    size_t cap = 0;
    int reserve(cmd_engine *eng, size_t bytes);
    void release(cmd_engine *eng);
};

// Growable pinned host buffer (staging for host-pointer calls).
struct HostScratch {
    void *ptr = nullptr;
    size_t cap = 0;
    int reserve(size_t bytes);
    void release();
};

// Fused-kernel launch configuration chosen per parameter set.
struct FusedConfig {
    int wpb = 8;          // warps per CTA (4 or 8)
    bool balanced = true; // equal-share rounds (see round_size in batch.cu)
    bool tuned = false;
    double ns_per_ct = 0; // measured by the tuner
    uint32_t tile_below = 0;  // CMD_PATH_AUTO: batches smaller than this take
                              // the tile kernels (five warps per 32-ciphertext
                              // tile for Berlekamp-Massey, one warp per
                              // ciphertext for the FFTs) instead of the fused
                              // kernel (one warp per tile); 0 = never
};

int cuda_fail(cudaError_t e, const char *what);
// T of the public key [I | T] of a key, from its device support d_L (n
// entries) and Goppa polynomial d_g (t + 1 coefficients): column c at
// d_cols[c * cwp ..], cwp >= ceil(mt / 32) words.  CMD_E_ARG when the key's
// parity-check matrix has no systematic form.  Takes eng->mu.
int kg_pubkey_columns(cmd_engine *eng, int set, const uint16_t *d_L, const uint16_t *d_g, uint32_t *d_cols, int cwp);
bool valid_set(int set);
bool budget_take(cmd_engine *eng, size_t bytes);
// Device address of GPU-mapped host memory [h, h + bytes) (2-byte aligned,
// one contiguous mapping), or null.
uint8_t *device_view(uint8_t *h, size_t bytes);
void budget_give(cmd_engine *eng, size_t bytes);

int run_device(cmd_engine *eng, const cmd_key *key, cmd_path path, const uint8_t *d_cts, size_t count,
               uint32_t *d_err, uint16_t *d_weight, cudaStream_t s);
int run_fused_single(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                     uint16_t *d_weight, cudaStream_t s, uint16_t *d_pos = nullptr);
// Explicit work counter and round schedule (balanced: -1 = the tuned choice,
// 0 = full rounds, 1 = equal shares; round_cts > 0 overrides all three with
// rounds of that many ciphertexts, a multiple of 32 from fused_round).
// err_packed: or null, a device-writable view of rows of n/8 bytes back to
// back (a host-mapped buffer the kernel fills directly).
int run_fused_counter(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                      uint16_t *d_weight, cudaStream_t s, uint32_t *counter, uint16_t *d_pos, int balanced,
                      uint32_t round_cts = 0, uint8_t *err_packed = nullptr);
// Ciphertexts per round of one launch over `count` ciphertexts of `set` under
// the tuned schedule.
uint32_t fused_round(cmd_engine *eng, int set, size_t count);
int ensure_counter(cmd_engine *eng);  // eng->tile_counter: 64 u32 work counters
constexpr int BATCH_STREAMS = 8;      // pieces of a host-buffer batch in flight
size_t fused_smem(int set, int wpb);
size_t smem_limit_bytes();
int fused_blocks_per_sm(int single_set, int wpb, size_t smem);
int fused_grid(cmd_engine *eng, int single_set, int wpb, size_t smem, uint64_t rounds);
int mixed_single_set(const int *key_set, const uint32_t *key_idx, size_t count);
void plan_mixed(const int *key_set, size_t nkeys, const uint32_t *key_idx, size_t count, uint32_t R,
                std::vector<uint32_t> &order, std::vector<FusedTile> &tiles);
// Root-search tables (fft_plan.cpp): uploaded once per engine, budget-charged.
int upload_fft_plans(cmd_engine *eng);
// No-allocation path (noalloc.cu): with `device` current, looks up the
// scratch array's device address and loads the plain kernels, so that
// cmd_decrypt_plain_noalloc itself loads and allocates nothing.
int noalloc_setup(int device);
void release_fft_plans(cmd_engine *eng);
inline FusedKeyRef key_ref(const KeyDev &k) { return FusedKeyRef{k.set, 0, k.tabd, k.Lbs, k.bctl}; }

}  // namespace cmd

struct cmd_engine {
    int device = 0;
    int num_sms = 0;
    char gpu_name[256] = {0};
    size_t budget = 0;
    std::atomic<size_t> used{0};
    cudaStream_t stream = nullptr;
    std::mutex mu;                 // serialises calls that share scratch
    cmd::Scratch scratch;          // plain-path intermediates
    cmd::Scratch io;               // device staging for host-buffer calls
    cmd::Scratch fused;            // fused-kernel work lists
    cmd::Scratch keygen;           // key-generation workspace (kept between calls)
    cmd::HostScratch host_scratch; // pinned staging
    uint32_t *tile_counter = nullptr;
    cudaStream_t piece_stream[cmd::BATCH_STREAMS] = {};  // host-buffer batches, created on first use
    std::atomic<uint64_t> launches{0};
    cmd::FusedConfig fcfg[cmd::NSETS];
    cmd::FusedConfig fcfg_mixed;
    cmd::FftPlanDev fft[cmd::NSETS] = {};  // per-set root-search tables
    void *fft_mem = nullptr;
    size_t fft_bytes = 0;
};

namespace cmd {
inline void fill_fft(FusedArgs &a, const cmd_engine *eng)
{
    for (int s = 0; s < NSETS; s++)
        a.fft[s] = eng->fft[s];
}
}  // namespace cmd

struct cmd_key {
    cmd_engine *eng = nullptr;
    cmd::KeyDev dev;
    void *block = nullptr;
    size_t bytes = 0;
    uint32_t *pk = nullptr;  // decapsulation: T block of the public key, column-major
    size_t pk_bytes = 0;
    std::mutex prep_mu;      // cmd_key_prepare_decap, per key (before eng->mu)
};
