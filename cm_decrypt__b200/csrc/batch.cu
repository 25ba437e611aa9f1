// Host side of the fused path: round lists for single-key and mixed batches,
// the persistent-grid sizing, and the pinned staging buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "engine.h"

namespace cmd {

int fused_blocks_per_sm(int single_set, int wpb, size_t smem);

int HostScratch::reserve(size_t bytes)
{
    if (bytes <= cap)
        return CMD_OK;
    if (ptr)
        cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost(&ptr, bytes);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMallocHost");
    cap = bytes;
    return CMD_OK;
}

void HostScratch::release()
{
    if (ptr)
        cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}

int ensure_counter(cmd_engine *eng)
{
    if (eng->tile_counter)
        return CMD_OK;
    cudaError_t e = cudaMalloc(&eng->tile_counter, 256);
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "cudaMalloc(counter)");
}

// Persistent grid: resident CTAs per SM (occupancy with this smem) x SMs,
// never more CTAs than rounds.
static int grid_for(cmd_engine *eng, int single_set, int wpb, size_t smem, uint64_t rounds)
{
    int per_sm = fused_blocks_per_sm(single_set, wpb, smem);
    if (per_sm < 1)
        per_sm = 1;
    uint64_t g = (uint64_t)per_sm * (uint64_t)eng->num_sms;
    return (int)std::min<uint64_t>(g, rounds);
}

// Ciphertexts per round.  `full` (every round fills all WPB warps) leaves
// the last wave partly idle when the batch is not a multiple of the resident
// capacity; `balanced` shrinks rounds (in whole 32-ciphertext tiles) so the
// batch splits into equal shares per resident CTA.
static uint32_t round_size(cmd_engine *eng, int set, int wpb, size_t count, bool balanced)
{
    const uint64_t full = (uint64_t)wpb * 32;
    if (!balanced)
        return (uint32_t)full;
    int per_sm = fused_blocks_per_sm(set, wpb, fused_smem(set, wpb));
    const uint64_t ctas = (uint64_t)(per_sm < 1 ? 1 : per_sm) * eng->num_sms;
    const uint64_t waves = (count + ctas * full - 1) / (ctas * full);
    uint64_t r = (count + ctas * waves - 1) / (ctas * waves);
    r = (r + 31) / 32 * 32;
    return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(r, 32), full);
}

uint32_t fused_round(cmd_engine *eng, int set, size_t count)
{
    return round_size(eng, set, eng->fcfg[set].wpb, count, eng->fcfg[set].balanced);
}

int run_fused_counter(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                      uint16_t *d_weight, cudaStream_t s, uint32_t *counter, uint16_t *d_pos, int balanced,
                      uint32_t round_cts, uint8_t *err_packed)
{
    const int set = key->dev.set;
    const SetInfo si = set_info(set);
    const int wpb = eng->fcfg[set].wpb;
    if (round_cts % 32 != 0 || round_cts > (uint32_t)wpb * 32) {
        set_last_error("fused round of " + std::to_string(round_cts) +
                       " ciphertexts: must be a multiple of 32 and at most " + std::to_string(wpb * 32));
        return CMD_E_ARG;
    }
    const uint32_t round = round_cts ? round_cts
                                     : round_size(eng, set, wpb, count,
                                                  balanced < 0 ? eng->fcfg[set].balanced : balanced != 0);
    const uint64_t rounds = (count + round - 1) / round;
    if (rounds > 0xFFFFFFFFull) {
        set_last_error("batch needs more than 2^32 fused rounds");
        return CMD_E_ARG;
    }
    FusedArgs a;
    memset(&a, 0, sizeof a);
    a.tiles = nullptr;
    a.ntiles = (uint32_t)rounds;
    a.round_cts = round;
    a.total = count;
    a.keys = nullptr;
    a.key0 = key_ref(key->dev);
    a.cts = d_cts;
    a.err = d_err;
    a.weight = d_weight;
    a.tile_counter = counter;
    a.single_set = set;
    fill_fft(a, eng);
    a.err_stride = (uint32_t)si.nw;
    a.pos = d_pos;
    a.pos_stride = (uint32_t)(si.t + 1);
    a.err_packed = err_packed;
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMemsetAsync(counter)");
    const int grid = grid_for(eng, set, wpb, fused_smem(set, wpb), rounds);
    e = launch_fused(a, grid, wpb, s, LaunchCounter{&eng->launches});
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "fused kernel launch");
}

// Sets the fused kernel's shared-memory attribute for this set's current
// configuration ahead of time (e.g. before a stream capture begins).
cudaError_t fused_prepare(cmd_engine *eng, int set)
{
    const int wpb = eng->fcfg[set].wpb;
    return fused_blocks_per_sm(set, wpb, fused_smem(set, wpb)) > 0 ? cudaSuccess : cudaErrorInvalidConfiguration;
}

int run_fused_single(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                     uint16_t *d_weight, cudaStream_t s, uint16_t *d_pos)
{
    int rc = ensure_counter(eng);
    if (rc)
        return rc;
    return run_fused_counter(eng, key, d_cts, count, d_err, d_weight, s, eng->tile_counter, d_pos, -1);
}

// Set shared by every ciphertext of a mixed batch, or -1.
int mixed_single_set(const int *key_set, const uint32_t *key_idx, size_t count)
{
    if (count == 0)
        return -1;
    const int s0 = key_set[key_idx[0]];
    for (size_t c = 1; c < count; c++)
        if (key_set[key_idx[c]] != s0)
            return -1;
    return s0;
}

// Groups ciphertexts by key (counting sort, stable in batch order) into
// `order` and cuts each key's run into rounds of up to R; rounds of costlier
// sets come first so the dynamic scheduler ends with cheap rounds.
void plan_mixed(const int *key_set, size_t nkeys, const uint32_t *key_idx, size_t count, uint32_t R,
                std::vector<uint32_t> &order, std::vector<FusedTile> &tiles)
{
    std::vector<uint32_t> cnt(nkeys + 1, 0);
    for (size_t c = 0; c < count; c++)
        cnt[key_idx[c] + 1]++;
    for (size_t k = 0; k < nkeys; k++)
        cnt[k + 1] += cnt[k];
    order.assign(count, 0);
    std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1);
    for (size_t c = 0; c < count; c++)
        order[fill[key_idx[c]]++] = (uint32_t)c;
    tiles.clear();
    for (size_t k = 0; k < nkeys; k++)
        for (uint32_t r0 = cnt[k]; r0 < cnt[k + 1]; r0 += R)
            tiles.push_back(FusedTile{(uint32_t)k, std::min(R, cnt[k + 1] - r0), r0});
    auto cost = [&](const FusedTile &t) {
        const SetInfo si = set_info(key_set[t.key]);
        return (uint64_t)si.n * si.t * si.m * si.m;
    };
    std::stable_sort(tiles.begin(), tiles.end(),
                     [&](const FusedTile &x, const FusedTile &y) { return cost(x) > cost(y); });
}

int fused_grid(cmd_engine *eng, int single_set, int wpb, size_t smem, uint64_t rounds)
{
    return grid_for(eng, single_set, wpb, smem, rounds);
}

}  // namespace cmd

using namespace cmd;

extern "C" int cmd_decrypt_mixed_device(cmd_engine *eng, const cmd_key *const *keys, size_t nkeys,
                                        const uint32_t *h_key_idx, const uint8_t *d_cts, const uint64_t *h_ct_off,
                                        size_t count, uint32_t *d_err, const uint64_t *h_err_off,
                                        uint16_t *d_weight, void *stream)
{
    if (!eng || (count && (!keys || !nkeys || !h_key_idx || !d_cts || !h_ct_off || !d_err || !h_err_off)))
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    if (count > 0xFFFFFFFFull || nkeys > 0xFFFFFFFFull) {
        set_last_error("mixed batch: more than 2^32 ciphertexts or keys");
        return CMD_E_ARG;
    }
    for (size_t k = 0; k < nkeys; k++)
        if (!keys[k] || keys[k]->eng != eng) {
            set_last_error("mixed batch: key " + std::to_string(k) + " is null or belongs to another engine");
            return CMD_E_ARG;
        }
    cudaSetDevice(eng->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;

    for (size_t c = 0; c < count; c++)
        if (h_key_idx[c] >= nkeys) {
            set_last_error("mixed batch: ciphertext " + std::to_string(c) + " names key " +
                           std::to_string(h_key_idx[c]) + " of " + std::to_string(nkeys));
            return CMD_E_ARG;
        }
    std::vector<int> kset(nkeys);
    for (size_t k = 0; k < nkeys; k++)
        kset[k] = keys[k]->dev.set;
    int single = mixed_single_set(kset.data(), h_key_idx, count);
    const int wpb = single >= 0 ? eng->fcfg[single].wpb : eng->fcfg_mixed.wpb;
    std::vector<uint32_t> order;
    std::vector<FusedTile> tiles;
    plan_mixed(kset.data(), nkeys, h_key_idx, count, (uint32_t)wpb * 32, order, tiles);
    std::vector<FusedKeyRef> krefs(nkeys);
    for (size_t k = 0; k < nkeys; k++)
        krefs[k] = key_ref(keys[k]->dev);

    std::lock_guard<std::mutex> lk(eng->mu);
    int rc = 0;
    if ((rc = [&] {
            if (eng->tile_counter)
                return CMD_OK;
            cudaError_t e = cudaMalloc(&eng->tile_counter, 256);
            return e == cudaSuccess ? CMD_OK : cuda_fail(e, "cudaMalloc(counter)");
        }()))
        return rc;
    // One device block for the work lists; pageable sources, so each copy has
    // consumed its host buffer when cudaMemcpyAsync returns.
    const size_t b_order = count * 4, b_off = count * 8, b_tiles = tiles.size() * sizeof(FusedTile),
                 b_keys = nkeys * sizeof(FusedKeyRef);
    auto al = [](size_t x) { return (x + 255) / 256 * 256; };
    const size_t need = al(b_order) + 2 * al(b_off) + al(b_tiles) + al(b_keys);
    if ((rc = eng->fused.reserve(eng, need)))
        return rc;
    uint8_t *base = static_cast<uint8_t *>(eng->fused.ptr);
    uint32_t *d_order = reinterpret_cast<uint32_t *>(base);
    uint64_t *d_ct_off = reinterpret_cast<uint64_t *>(base + al(b_order));
    uint64_t *d_err_off = reinterpret_cast<uint64_t *>(base + al(b_order) + al(b_off));
    FusedTile *d_tiles = reinterpret_cast<FusedTile *>(base + al(b_order) + 2 * al(b_off));
    FusedKeyRef *d_keys = reinterpret_cast<FusedKeyRef *>(base + al(b_order) + 2 * al(b_off) + al(b_tiles));
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_order, order.data(), b_order, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_ct_off, h_ct_off, b_off, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_err_off, h_err_off, b_off, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_tiles, tiles.data(), b_tiles, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_keys, krefs.data(), b_keys, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(eng->tile_counter, 0, sizeof(uint32_t), s)) != cudaSuccess)
        return cuda_fail(e, "mixed batch upload");
    FusedArgs a;
    memset(&a, 0, sizeof a);
    a.tiles = d_tiles;
    a.ntiles = (uint32_t)tiles.size();
    a.keys = d_keys;
    a.cts = d_cts;
    a.ct_off = d_ct_off;
    a.err_off = d_err_off;
    a.order = d_order;
    a.err = d_err;
    a.weight = d_weight;
    a.tile_counter = eng->tile_counter;
    a.single_set = single;
    fill_fft(a, eng);
    size_t smem = 0;
    if (single >= 0)
        smem = fused_smem(single, wpb);
    else
        for (int st = 0; st < NSETS; st++)
            smem = std::max(smem, fused_smem(st, wpb));
    const int grid = grid_for(eng, single, wpb, smem, tiles.size());
    e = launch_fused(a, grid, wpb, s, LaunchCounter{&eng->launches});
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "fused kernel launch (mixed)");
}
