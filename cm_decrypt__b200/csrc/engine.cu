// C ABI of the decryption engine (include/cmd_b200.h): engine and key
// lifetime, the HBM budget, batch scheduling over the plain and fused kernel
// paths, and the host<->device staging for host-buffer calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "engine.h"

namespace cmd {
static int run_tile(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                    uint16_t *d_weight, uint16_t *d_synd, cudaStream_t s);

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }

int cuda_fail(cudaError_t e, const char *what)
{
    set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
    return CMD_E_CUDA;
}

bool valid_set(int set) { return set >= 0 && set < NSETS; }

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Charges `bytes` against the engine budget; false if it would not fit.
bool budget_take(cmd_engine *eng, size_t bytes)
{
    size_t cur = eng->used.load();
    while (true) {
        if (cur + bytes > eng->budget)
            return false;
        if (eng->used.compare_exchange_weak(cur, cur + bytes))
            return true;
    }
}
void budget_give(cmd_engine *eng, size_t bytes) { eng->used.fetch_sub(bytes); }

int Scratch::reserve(cmd_engine *eng, size_t bytes)
{
    if (bytes <= cap)
        return CMD_OK;
    size_t want = align_up(std::max(bytes, cap + cap / 2), 1 << 20);
    if (!budget_take(eng, want - cap)) {
        set_last_error("scratch growth exceeds the engine HBM budget");
        return CMD_E_BUDGET;
    }
    if (ptr) {
        cudaFree(ptr);
        ptr = nullptr;
    }
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) {
        budget_give(eng, want - cap);
        budget_give(eng, cap);
        cap = 0;
        return cuda_fail(e, "cudaMalloc(scratch)");
    }
    cap = want;
    return CMD_OK;
}

void Scratch::release(cmd_engine *eng)
{
    if (ptr)
        cudaFree(ptr);
    budget_give(eng, cap);
    ptr = nullptr;
    cap = 0;
}

// Bump allocation inside one scratch reservation (256-byte aligned slices).
struct Carver {
    uint8_t *base;
    size_t off = 0;
    template <class T> T *take(size_t count)
    {
        off = align_up(off, 256);
        T *p = reinterpret_cast<T *>(base + off);
        off += count * sizeof(T);
        return p;
    }
};
static size_t carve_size(std::initializer_list<size_t> sizes)
{
    size_t off = 0;
    for (size_t s : sizes)
        off = align_up(off, 256) + s;
    return off + 256;
}

}  // namespace cmd

using namespace cmd;

extern "C" {

const char *cmd_last_error(void) { return g_last_error.c_str(); }

int cmd_set_info_get(cmd_set set, cmd_set_info *out)
{
    if (!out || !valid_set(set))
        return CMD_E_ARG;
    SetInfo s = set_info(set);
    out->set_id = s.id;
    out->m = s.m;
    out->n = s.n;
    out->t = s.t;
    out->ct_bytes = s.ct;
    out->sk_bytes = s.sk;
    out->sb = s.sb;
    out->err_bytes = s.n / 8;
    out->err_words = s.nw;
    return CMD_OK;
}

int cmd_set_from_name(const char *name, cmd_set *out)
{
    if (!name || !out)
        return CMD_E_ARG;
    const char *p = name;
    if (!strncmp(p, "mceliece", 8))
        p += 8;
    for (int s = 0; s < NSETS; s++) {
        char buf[16];
        snprintf(buf, sizeof buf, "%d", set_info(s).id);
        if (!strcmp(p, buf)) {
            *out = (cmd_set)s;
            return CMD_OK;
        }
    }
    set_last_error(std::string("unknown parameter set: ") + name);
    return CMD_E_ARG;
}

int cmd_engine_create(int device, size_t hbm_budget_bytes, cmd_engine **out)
{
    if (!out)
        return CMD_E_ARG;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device");
        return CMD_E_NODEVICE;
    }
    if (device < 0 || device >= ndev)
        return CMD_E_ARG;
    if ((e = cudaSetDevice(device)) != cudaSuccess)
        return cuda_fail(e, "cudaSetDevice");
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess)
        return cuda_fail(e, "cudaGetDeviceProperties");
    if (prop.major != 10) {
        set_last_error("this build targets sm_100a (B200); device is sm_" + std::to_string(prop.major) +
                       std::to_string(prop.minor));
        return CMD_E_NODEVICE;
    }
    cmd_engine *eng = new (std::nothrow) cmd_engine();
    if (!eng)
        return CMD_E_NOMEM;
    eng->device = device;
    eng->num_sms = prop.multiProcessorCount;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    eng->budget = hbm_budget_bytes ? hbm_budget_bytes : free_b / 10 * 8;
    if ((e = cudaStreamCreateWithFlags(&eng->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        delete eng;
        return cuda_fail(e, "cudaStreamCreate");
    }
    snprintf(eng->gpu_name, sizeof eng->gpu_name, "%s", prop.name);
    if (int rc = noalloc_setup(device)) {
        cudaStreamDestroy(eng->stream);
        delete eng;
        return rc;
    }
    if (int rc = upload_fft_plans(eng)) {
        cudaStreamDestroy(eng->stream);
        delete eng;
        return rc;
    }
    *out = eng;
    return CMD_OK;
}

void cmd_engine_destroy(cmd_engine *eng)
{
    if (!eng)
        return;
    cudaSetDevice(eng->device);
    cudaStreamSynchronize(eng->stream);
    eng->scratch.release(eng);
    eng->io.release(eng);
    eng->fused.release(eng);
    eng->keygen.release(eng);
    eng->host_scratch.release();
    release_fft_plans(eng);
    for (int i = 0; i < BATCH_STREAMS; i++)
        if (eng->piece_stream[i]) {
            cudaStreamSynchronize(eng->piece_stream[i]);
            cudaStreamDestroy(eng->piece_stream[i]);
        }
    if (eng->tile_counter)
        cudaFree(eng->tile_counter);
    cudaStreamDestroy(eng->stream);
    delete eng;
}

int cmd_engine_memory(const cmd_engine *eng, size_t *used, size_t *budget)
{
    if (!eng)
        return CMD_E_ARG;
    if (used)
        *used = eng->used.load();
    if (budget)
        *budget = eng->budget;
    return CMD_OK;
}

uint64_t cmd_engine_launch_count(const cmd_engine *eng) { return eng ? eng->launches.load() : 0; }

// ---------------------------------------------------------------- keys

int cmd_key_expand(cmd_engine *eng, cmd_set set, const uint8_t *h_sk, size_t sk_len, cmd_key **out)
{
    if (!eng || !h_sk || !out || !valid_set(set))
        return CMD_E_ARG;
    *out = nullptr;
    const SetInfo si = set_info(set);
    if (sk_len != (size_t)si.sk) {
        set_last_error("secret key must be exactly " + std::to_string(si.sk) + " bytes for set " +
                       std::to_string(si.id));
        return CMD_E_ARG;
    }
    const size_t bytes = carve_size({(size_t)si.n * 2, (size_t)(si.t + 1) * 2, (size_t)si.n * 2,
                                     (size_t)si.sb * si.twp() * 4, (size_t)si.sb * si.twd() * 4,
                                     (size_t)si.m * si.nw * 4,
                                     benes_mask_words(si) * 4, fft_weight_words(si) * 4, (size_t)si.sk});
    if (!budget_take(eng, bytes)) {
        set_last_error("key does not fit the engine HBM budget");
        return CMD_E_BUDGET;
    }
    cmd_key *key = new (std::nothrow) cmd_key();
    if (!key) {
        budget_give(eng, bytes);
        return CMD_E_NOMEM;
    }
    key->eng = eng;
    key->bytes = bytes;
    cudaSetDevice(eng->device);
    cudaError_t e = cudaMalloc(&key->block, bytes);
    if (e != cudaSuccess) {
        budget_give(eng, bytes);
        delete key;
        return cuda_fail(e, "cudaMalloc(key)");
    }
    Carver cv{static_cast<uint8_t *>(key->block)};
    key->dev.set = set;
    key->dev.L = cv.take<uint16_t>(si.n);
    key->dev.g = cv.take<uint16_t>(si.t + 1);
    key->dev.ginv2 = cv.take<uint16_t>(si.n);
    key->dev.tab = cv.take<uint32_t>((size_t)si.sb * si.twp());
    key->dev.tabd = cv.take<uint32_t>((size_t)si.sb * si.twd());
    key->dev.Lbs = cv.take<uint32_t>((size_t)si.m * si.nw);
    key->dev.bctl = cv.take<uint32_t>(benes_mask_words(si));
    key->dev.wfft = cv.take<uint32_t>(fft_weight_words(si));
    key->dev.sk = cv.take<uint8_t>(si.sk);
    std::lock_guard<std::mutex> lk(eng->mu);
    if ((e = cudaMemcpyAsync(key->dev.sk, h_sk, si.sk, cudaMemcpyHostToDevice, eng->stream)) != cudaSuccess ||
        (e = launch_key_expand(key->dev, eng->stream, LaunchCounter{&eng->launches})) != cudaSuccess ||
        (e = cudaStreamSynchronize(eng->stream)) != cudaSuccess) {
        cudaFree(key->block);
        budget_give(eng, bytes);
        delete key;
        return cuda_fail(e, "key expansion");
    }
    *out = key;
    return CMD_OK;
}

void cmd_key_free(cmd_key *key)
{
    if (!key)
        return;
    cudaSetDevice(key->eng->device);
    cudaStreamSynchronize(key->eng->stream);
    cudaFree(key->block);
    budget_give(key->eng, key->bytes);
    if (key->pk) {
        cudaFree(key->pk);
        budget_give(key->eng, key->pk_bytes);
    }
    delete key;
}

int cmd_key_set(const cmd_key *key, cmd_set *out)
{
    if (!key || !out)
        return CMD_E_ARG;
    *out = (cmd_set)key->dev.set;
    return CMD_OK;
}

size_t cmd_key_device_bytes(const cmd_key *key) { return key ? key->bytes : 0; }

static int key_copy(const cmd_key *key, void *dst, const void *src, size_t bytes)
{
    cudaSetDevice(key->eng->device);
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "cudaMemcpy(key D2H)");
}

int cmd_key_support(const cmd_key *key, uint16_t *h_L, size_t n)
{
    if (!key || !h_L || n != (size_t)set_info(key->dev.set).n)
        return CMD_E_ARG;
    return key_copy(key, h_L, key->dev.L, n * 2);
}

int cmd_key_goppa(const cmd_key *key, uint16_t *h_g, size_t t_plus_1)
{
    if (!key || !h_g || t_plus_1 != (size_t)set_info(key->dev.set).t + 1)
        return CMD_E_ARG;
    return key_copy(key, h_g, key->dev.g, t_plus_1 * 2);
}

int cmd_key_synd_table(const cmd_key *key, uint16_t *h_tab, size_t entries)
{
    const SetInfo si = key ? set_info(key->dev.set) : SetInfo{};
    if (!key || !h_tab || entries != (size_t)si.sb * 2 * si.t)
        return CMD_E_ARG;
    cudaSetDevice(key->eng->device);
    cudaError_t e = cudaMemcpy2D(h_tab, (size_t)si.t * 4, key->dev.tab, (size_t)si.twp() * 4, (size_t)si.t * 4,
                                 si.sb, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "cudaMemcpy2D(table D2H)");
}

// ---------------------------------------------------------------- stages

int cmd_stage_synd(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint16_t *d_synd,
                   void *stream)
{
    if (!eng || !key || (count && (!d_cts || !d_synd)))
        return CMD_E_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    cudaError_t e = launch_synd_plain(key->dev, d_cts, count, reinterpret_cast<uint32_t *>(d_synd), s,
                                      LaunchCounter{&eng->launches});
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "synd kernel");
}

int cmd_stage_synd_fft(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint16_t *d_synd,
                       void *stream)
{
    if (!eng || !key || key->eng != eng || (count && (!d_cts || !d_synd)))
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    cudaSetDevice(eng->device);
    std::lock_guard<std::mutex> lk(eng->mu);
    return run_tile(eng, key, d_cts, count, nullptr, nullptr, d_synd, stream ? (cudaStream_t)stream : eng->stream);
}

int cmd_stage_bm(cmd_engine *eng, cmd_set set, const uint16_t *d_synd, size_t count, uint16_t *d_loc, void *stream)
{
    if (!eng || !valid_set(set) || (count && (!d_synd || !d_loc)))
        return CMD_E_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    cudaError_t e = launch_bm_plain(set, d_synd, count, d_loc, s, LaunchCounter{&eng->launches});
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "bm kernel");
}

int cmd_stage_root(cmd_engine *eng, const cmd_key *key, const uint16_t *d_loc, size_t count, uint32_t *d_err,
                   uint16_t *d_weight, void *stream)
{
    if (!eng || !key || (count && (!d_loc || !d_err)))
        return CMD_E_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    cudaError_t e = launch_root_plain(key->dev, d_loc, count, d_err, d_weight, s, LaunchCounter{&eng->launches},
                                      eng->num_sms);
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "root kernel");
}

int cmd_stage_root_images(cmd_engine *eng, const cmd_key *key, const uint16_t *d_loc, size_t count,
                          uint16_t *d_images, void *stream)
{
    if (!eng || !key || (count && (!d_loc || !d_images)))
        return CMD_E_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    cudaError_t e = launch_root_images(key->dev, d_loc, count, d_images, s, LaunchCounter{&eng->launches});
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "root images kernel");
}

// ---------------------------------------------------------------- batches

}  // extern "C"

namespace cmd {

// Scratch the plain path needs for a batch: per chunk of up to 2^18
// ciphertexts, the syndromes (t words) and locators (t+1 u16) of each.
size_t plain_scratch_bytes(int set, size_t count)
{
    const SetInfo si = set_info(set);
    const size_t chunk = std::min<size_t>(count, (size_t)1 << 18);
    return carve_size({chunk * si.t * 4, chunk * (si.t + 1) * 2});
}

// Plain path over a device batch, in chunks so the syndrome/locator
// intermediates stay bounded.  Caller holds eng->mu.
static int run_plain(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                     uint16_t *d_weight, cudaStream_t s)
{
    const SetInfo si = set_info(key->dev.set);
    const size_t chunk = std::min<size_t>(count, (size_t)1 << 18);
    const size_t need = plain_scratch_bytes(key->dev.set, count);
    int rc = eng->scratch.reserve(eng, need);
    if (rc)
        return rc;
    Carver cv{static_cast<uint8_t *>(eng->scratch.ptr)};
    uint32_t *synd = cv.take<uint32_t>(chunk * si.t);
    uint16_t *loc = cv.take<uint16_t>(chunk * (si.t + 1));
    LaunchCounter lc{&eng->launches};
    for (size_t c0 = 0; c0 < count; c0 += chunk) {
        const size_t n = std::min(chunk, count - c0);
        cudaError_t e;
        if ((e = launch_synd_plain(key->dev, d_cts + c0 * si.ct, n, synd, s, lc)) != cudaSuccess ||
            (e = launch_bm_plain(key->dev.set, reinterpret_cast<uint16_t *>(synd), n, loc, s, lc)) != cudaSuccess ||
            (e = launch_root_plain(key->dev, loc, n, d_err + c0 * si.nw, d_weight ? d_weight + c0 : nullptr, s, lc,
                                   eng->num_sms)) != cudaSuccess)
            return cuda_fail(e, "plain path launch");
    }
    return CMD_OK;
}

// The serving tile kernels over one key's batch, in chunks whose byte and
// word offsets fit the tile items' 32-bit fields.  With d_synd: syndromes
// only.  Caller holds eng->mu.
static int run_tile(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                    uint16_t *d_weight, uint16_t *d_synd, cudaStream_t s)
{
    const SetInfo si = set_info(key->dev.set);
    const size_t chunk = std::min<size_t>(count, (size_t)1 << 22);
    int rc = eng->scratch.reserve(eng, tile_single_scratch_words(chunk) * 4);
    if (rc)
        return rc;
    FftPlans plans;
    for (int st = 0; st < NSETS; st++)
        plans.p[st] = eng->fft[st];
    for (size_t c0 = 0; c0 < count; c0 += chunk) {
        const size_t n = std::min(chunk, count - c0);
        const cudaError_t e = launch_tile_single(
            key->dev, d_cts + c0 * si.ct, n, static_cast<uint32_t *>(eng->scratch.ptr),
            d_err ? d_err + c0 * si.nw : nullptr, d_weight ? d_weight + c0 : nullptr,
            d_synd ? d_synd + c0 * 2 * si.t : nullptr, plans, s, LaunchCounter{&eng->launches});
        if (e != cudaSuccess)
            return cuda_fail(e, "tile path launch");
    }
    return CMD_OK;
}

int run_device(cmd_engine *eng, const cmd_key *key, cmd_path path, const uint8_t *d_cts, size_t count,
               uint32_t *d_err, uint16_t *d_weight, cudaStream_t s)
{
    if (count == 0)
        return CMD_OK;
    if (path == CMD_PATH_PLAIN)
        return run_plain(eng, key, d_cts, count, d_err, d_weight, s);
    if (path == CMD_PATH_TILE || (path == CMD_PATH_AUTO && count < eng->fcfg[key->dev.set].tile_below))
        return run_tile(eng, key, d_cts, count, d_err, d_weight, nullptr, s);
    return run_fused_single(eng, key, d_cts, count, d_err, d_weight, s);
}

// A device address through which kernels can write the host range [h, h +
// bytes), or null: pinned memory the GPU maps (cudaHostAlloc / cudaMallocHost
// memory under unified addressing, or registered memory with a device
// mapping), 2-byte aligned, whose first and last bytes map to one contiguous
// device range.  Anything else (pageable memory, a range running past its
// pinned allocation) gives null, and the caller copies through staging.
uint8_t *device_view(uint8_t *h, size_t bytes)
{
    if (!h || !bytes || (((uintptr_t)h) & 1))
        return nullptr;
    cudaPointerAttributes a0{}, a1{};
    if (cudaPointerGetAttributes(&a0, h) != cudaSuccess || a0.type != cudaMemoryTypeHost || !a0.devicePointer) {
        cudaGetLastError();
        return nullptr;
    }
    if (cudaPointerGetAttributes(&a1, h + bytes - 1) != cudaSuccess || a1.type != cudaMemoryTypeHost ||
        static_cast<uint8_t *>(a1.devicePointer) != static_cast<uint8_t *>(a0.devicePointer) + (bytes - 1)) {
        cudaGetLastError();
        return nullptr;
    }
    return static_cast<uint8_t *>(a0.devicePointer);
}

}  // namespace cmd

extern "C" {

int cmd_decrypt_device(cmd_engine *eng, const cmd_key *key, cmd_path path, const uint8_t *d_cts, size_t count,
                       uint32_t *d_err, uint16_t *d_weight, void *stream)
{
    if (!eng || !key || key->eng != eng || (count && (!d_cts || !d_err)) || path < 0 || path > 3)
        return CMD_E_ARG;
    cudaSetDevice(eng->device);
    std::lock_guard<std::mutex> lk(eng->mu);
    return run_device(eng, key, path, d_cts, count, d_err, d_weight, stream ? (cudaStream_t)stream : eng->stream);
}


int cmd_decrypt_batch(cmd_engine *eng, const cmd_key *key, cmd_path path, const uint8_t *h_cts, size_t count,
                      uint8_t *h_err, uint16_t *h_weight)
{
    if (!eng || !key || key->eng != eng || (count && (!h_cts || !h_err)) || path < 0 || path > 3)
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    cudaSetDevice(eng->device);
    const SetInfo si = set_info(key->dev.set);
    std::lock_guard<std::mutex> lk(eng->mu);
    // Device staging: ciphertexts, error rows, weights; processed in chunks so
    // the staging stays bounded for very large host batches.
    const size_t chunk = std::min<size_t>(count, (size_t)1 << 20);
    const size_t need = carve_size({chunk * si.ct, chunk * si.nw * 4, chunk * 2});
    int rc = eng->io.reserve(eng, need);
    if (rc)
        return rc;
    Carver cv{static_cast<uint8_t *>(eng->io.ptr)};
    uint8_t *d_cts = cv.take<uint8_t>(chunk * si.ct);
    uint32_t *d_err = cv.take<uint32_t>(chunk * si.nw);
    uint16_t *d_w = cv.take<uint16_t>(chunk);
    cudaStream_t s = eng->stream;
    // Large fused batches go as BATCH_STREAMS pieces on their own streams
    // (each with its own work counter, full rounds): one piece's copies run
    // while the others compute, and the pieces' kernels share the SMs.
    const bool pieces = path != CMD_PATH_PLAIN && path != CMD_PATH_TILE && chunk >= (size_t)BATCH_STREAMS * 8192;
    // With host error rows the GPU can write, the pieces' kernels store the
    // packed rows there directly: the rows cross PCIe while the kernels run,
    // instead of in a copy after the last piece's kernel.
    uint8_t *err_view = pieces ? device_view(h_err, count * (size_t)(si.n / 8)) : nullptr;
    if (pieces) {
        if ((rc = ensure_counter(eng)))
            return rc;
        for (int i = 0; i < BATCH_STREAMS; i++)
            if (!eng->piece_stream[i]) {
                cudaError_t e = cudaStreamCreateWithFlags(&eng->piece_stream[i], cudaStreamNonBlocking);
                if (e != cudaSuccess)
                    return cuda_fail(e, "cudaStreamCreate(piece)");
            }
    }
    for (size_t c0 = 0; c0 < count; c0 += chunk) {
        const size_t n = std::min(chunk, count - c0);
        if (pieces) {
            // pieces of whole rounds of the size one launch over the chunk
            // would use (equal shares per resident CTA when so tuned), so the
            // pieces' rounds fill the same waves; a round is a multiple of 32
            // ciphertexts, so every piece's ciphertexts start 16-byte aligned
            const uint32_t round = fused_round(eng, key->dev.set, n);
            const size_t per = (n + (size_t)BATCH_STREAMS * round - 1) / ((size_t)BATCH_STREAMS * round) * round;
            cudaError_t e = cudaSuccess;
            for (int i = 0; i < BATCH_STREAMS && e == cudaSuccess && rc == CMD_OK; i++) {
                const size_t p0 = (size_t)i * per;
                if (p0 >= n)
                    break;
                const size_t pn = std::min(per, n - p0);
                cudaStream_t ps = eng->piece_stream[i];
                e = cudaMemcpyAsync(d_cts + p0 * si.ct, h_cts + (c0 + p0) * si.ct, pn * si.ct, cudaMemcpyHostToDevice,
                                    ps);
                if (e != cudaSuccess)
                    break;
                uint8_t *pack = err_view ? err_view + (c0 + p0) * (size_t)(si.n / 8) : nullptr;
                rc = run_fused_counter(eng, key, d_cts + p0 * si.ct, pn, pack ? nullptr : d_err + p0 * si.nw,
                                       d_w + p0, ps, eng->tile_counter + 1 + i, nullptr, 0, round, pack);
                if (rc)
                    break;
                if (!pack)
                    e = cudaMemcpy2DAsync(h_err + (c0 + p0) * (si.n / 8), si.n / 8, d_err + p0 * si.nw,
                                          (size_t)si.nw * 4, si.n / 8, pn, cudaMemcpyDeviceToHost, ps);
                if (e == cudaSuccess && h_weight)
                    e = cudaMemcpyAsync(h_weight + c0 + p0, d_w + p0, pn * 2, cudaMemcpyDeviceToHost, ps);
            }
            for (int i = 0; i < BATCH_STREAMS; i++) {
                const cudaError_t e2 = cudaStreamSynchronize(eng->piece_stream[i]);
                if (e == cudaSuccess)
                    e = e2;
            }
            if (rc)
                return rc;
            if (e != cudaSuccess)
                return cuda_fail(e, "decrypt batch pieces");
            continue;
        }
        cudaError_t e = cudaMemcpyAsync(d_cts, h_cts + c0 * si.ct, n * si.ct, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(cts H2D)");
        if ((rc = run_device(eng, key, path, d_cts, n, d_err, d_w, s)))
            return rc;
        // Strip the word padding of each row: n/8 bytes per vector on the host.
        e = cudaMemcpy2DAsync(h_err + c0 * (si.n / 8), si.n / 8, d_err, (size_t)si.nw * 4, si.n / 8, n,
                              cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && h_weight)
            e = cudaMemcpyAsync(h_weight + c0, d_w, n * 2, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return cuda_fail(e, "decrypt batch D2H");
    }
    return CMD_OK;
}

int cmd_decrypt_positions_device(cmd_engine *eng, const cmd_key *key, const uint8_t *d_cts, size_t count,
                                 uint16_t *d_pos, void *stream)
{
    if (!eng || !key || key->eng != eng || (count && (!d_cts || !d_pos)))
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    cudaSetDevice(eng->device);
    std::lock_guard<std::mutex> lk(eng->mu);
    return run_fused_single(eng, key, d_cts, count, nullptr, nullptr, stream ? (cudaStream_t)stream : eng->stream,
                            d_pos);
}

int cmd_decrypt_positions(cmd_engine *eng, const cmd_key *key, const uint8_t *h_cts, size_t count, uint16_t *h_pos)
{
    if (!eng || !key || key->eng != eng || (count && (!h_cts || !h_pos)))
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    cudaSetDevice(eng->device);
    const SetInfo si = set_info(key->dev.set);
    const size_t row = (size_t)si.t + 1;
    std::lock_guard<std::mutex> lk(eng->mu);
    const size_t chunk = std::min<size_t>(count, (size_t)1 << 20);
    const size_t need = carve_size({chunk * si.ct, chunk * row * 2});
    int rc = eng->io.reserve(eng, need);
    if (rc)
        return rc;
    Carver cv{static_cast<uint8_t *>(eng->io.ptr)};
    uint8_t *d_cts = cv.take<uint8_t>(chunk * si.ct);
    uint16_t *d_pos = cv.take<uint16_t>(chunk * row);
    cudaStream_t s = eng->stream;
    const bool pieces = chunk >= (size_t)BATCH_STREAMS * 8192;
    if (pieces) {
        if ((rc = ensure_counter(eng)))
            return rc;
        for (int i = 0; i < BATCH_STREAMS; i++)
            if (!eng->piece_stream[i]) {
                cudaError_t e = cudaStreamCreateWithFlags(&eng->piece_stream[i], cudaStreamNonBlocking);
                if (e != cudaSuccess)
                    return cuda_fail(e, "cudaStreamCreate(piece)");
            }
    }
    for (size_t c0 = 0; c0 < count; c0 += chunk) {
        const size_t n = std::min(chunk, count - c0);
        if (pieces) {  // as in cmd_decrypt_batch
            const uint32_t round = fused_round(eng, key->dev.set, n);
            const size_t per = (n + (size_t)BATCH_STREAMS * round - 1) / ((size_t)BATCH_STREAMS * round) * round;
            cudaError_t e = cudaSuccess;
            for (int i = 0; i < BATCH_STREAMS && e == cudaSuccess && rc == CMD_OK; i++) {
                const size_t p0 = (size_t)i * per;
                if (p0 >= n)
                    break;
                const size_t pn = std::min(per, n - p0);
                cudaStream_t ps = eng->piece_stream[i];
                e = cudaMemcpyAsync(d_cts + p0 * si.ct, h_cts + (c0 + p0) * si.ct, pn * si.ct, cudaMemcpyHostToDevice,
                                    ps);
                if (e != cudaSuccess)
                    break;
                rc = run_fused_counter(eng, key, d_cts + p0 * si.ct, pn, nullptr, nullptr, ps,
                                       eng->tile_counter + 1 + i, d_pos + p0 * row, 0, round);
                if (rc)
                    break;
                e = cudaMemcpyAsync(h_pos + (c0 + p0) * row, d_pos + p0 * row, pn * row * 2, cudaMemcpyDeviceToHost,
                                    ps);
            }
            for (int i = 0; i < BATCH_STREAMS; i++) {
                const cudaError_t e2 = cudaStreamSynchronize(eng->piece_stream[i]);
                if (e == cudaSuccess)
                    e = e2;
            }
            if (rc)
                return rc;
            if (e != cudaSuccess)
                return cuda_fail(e, "decrypt positions pieces");
            continue;
        }
        cudaError_t e = cudaMemcpyAsync(d_cts, h_cts + c0 * si.ct, n * si.ct, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(cts H2D)");
        if ((rc = run_fused_single(eng, key, d_cts, n, nullptr, nullptr, s, d_pos)))
            return rc;
        e = cudaMemcpyAsync(h_pos + c0 * row, d_pos, n * row * 2, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return cuda_fail(e, "decrypt positions D2H");
    }
    return CMD_OK;
}

}  // extern "C"
