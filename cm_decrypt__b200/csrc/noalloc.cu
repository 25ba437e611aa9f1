// Allocation-free variant of the plain per-stage decrypt path.
//
// cmd_decrypt_device() keeps the plain path's intermediates (the 2t
// syndromes and the t+1 locator coefficients of every ciphertext) in engine
// scratch that grows with cudaMalloc.  Some callers cannot let a library do
// that: hosts whose device memory belongs to another allocator (a framework's
// memory pool that must see every byte), or latency-critical loops where a
// cudaMalloc/cudaFree and the device synchronisation it implies are not
// acceptable.  For them this file keeps the intermediates in one file-scope
// device array instead, sized for CMD_NOALLOC_MAX_CTS ciphertexts per call;
// every GPU that loads the library holds the array until the process exits.
//
// Host code cannot use the array's name as a device address (it names a host
// shadow), so cmd_engine_create, with the engine's device current, asks the
// runtime for the array's device address with cudaGetSymbolAddress and
// caches it per device.  With lazy module loading (the CUDA 12 default) that
// lookup is also what loads the array onto the device, and engine creation
// loads the plain kernels the same way, so the entry point itself neither
// loads a module nor allocates.  Calls share the array and it keeps the
// previous call's contents; the kernels overwrite every syndrome and locator
// entry they later read, so nothing needs clearing, but calls that overlap
// on the GPU (other streams or threads at the same time) race on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "engine.h"

namespace cmd {

// Per ciphertext: t (<= 128) syndrome words, then t+1 (<= 129) u16 locator
// coefficients; the largest set fixes both strides.
constexpr size_t NA_SYND_BYTES = (size_t)CMD_NOALLOC_MAX_CTS * 128 * 4;
constexpr size_t NA_LOC_BYTES = (size_t)CMD_NOALLOC_MAX_CTS * 129 * 2;
constexpr size_t NA_BYTES = NA_SYND_BYTES + NA_LOC_BYTES;

static __device__ __align__(256) uint8_t g_noalloc_scratch[NA_BYTES];

constexpr int NA_MAX_DEVICES = 64;
static std::mutex g_na_mu;
static void *g_na_ptr[NA_MAX_DEVICES];

// Called by cmd_engine_create with `device` current: the scratch array's
// device address (once per device) and the plain kernels' module.
int noalloc_setup(int device)
{
    if (device < 0 || device >= NA_MAX_DEVICES) {
        set_last_error("device index out of range for the no-alloc path");
        return CMD_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess)
            e = preload_plain_kernels();
        if (e != cudaSuccess)
            return cuda_fail(e, "no-alloc scratch set-up");
        g_na_ptr[device] = p;
    }
    return CMD_OK;
}

static uint8_t *noalloc_scratch(int device)
{
    if (device < 0 || device >= NA_MAX_DEVICES)
        return nullptr;
    std::lock_guard<std::mutex> lk(g_na_mu);
    return static_cast<uint8_t *>(g_na_ptr[device]);
}

}  // namespace cmd

using namespace cmd;

extern "C" int cmd_decrypt_plain_noalloc(const cmd_key *key, const uint8_t *d_cts, size_t count, uint32_t *d_err,
                                         uint16_t *d_weight, void *stream)
{
    if (!key || (count && (!d_cts || !d_err)))
        return CMD_E_ARG;
    if (count > CMD_NOALLOC_MAX_CTS) {
        set_last_error("cmd_decrypt_plain_noalloc: " + std::to_string(count) +
                       " ciphertexts exceed the per-call maximum of " + std::to_string(CMD_NOALLOC_MAX_CTS));
        return CMD_E_ARG;
    }
    if (count == 0)
        return CMD_OK;
    cmd_engine *eng = key->eng;
    uint8_t *base = noalloc_scratch(eng->device);
    if (!base) {
        set_last_error("no-alloc scratch not set up on this device (cmd_engine_create does it)");
        return CMD_E_ARG;
    }
    // the caller's current device is put back before returning
    int caller_dev = -1;
    cudaGetDevice(&caller_dev);
    if (caller_dev != eng->device)
        cudaSetDevice(eng->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    uint32_t *synd = reinterpret_cast<uint32_t *>(base);
    uint16_t *loc = reinterpret_cast<uint16_t *>(base + NA_SYND_BYTES);
    LaunchCounter lc{&eng->launches};
    cudaError_t e;
    int rc = CMD_OK;
    if ((e = launch_synd_plain(key->dev, d_cts, count, synd, s, lc)) != cudaSuccess ||
        (e = launch_bm_plain(key->dev.set, reinterpret_cast<uint16_t *>(synd), count, loc, s, lc)) != cudaSuccess ||
        (e = launch_root_plain(key->dev, loc, count, d_err, d_weight, s, lc, eng->num_sms)) != cudaSuccess)
        rc = cuda_fail(e, "no-alloc plain path launch");
    if (caller_dev >= 0 && caller_dev != eng->device)
        cudaSetDevice(caller_dev);
    return rc;
}
