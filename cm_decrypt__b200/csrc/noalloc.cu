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
// shadow), so the first call on each device, with that device current, asks
// the runtime for the array's device address with cudaGetSymbolAddress and
// caches it.  That first call should therefore be made before any stream
// capture begins.  Calls share the array and it keeps the previous call's
// contents; the kernels overwrite every syndrome and locator entry they later
// read, so nothing needs clearing, but calls that overlap on the GPU (other
// streams or threads at the same time) race on it.
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

// Device address of the scratch array on `device` (set up once per device).
static int noalloc_scratch(int device, uint8_t **out)
{
    if (device < 0 || device >= NA_MAX_DEVICES) {
        set_last_error("device index out of range for the no-alloc path");
        return CMD_E_ARG;
    }
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[device]) {
        int cur = -1;
        cudaGetDevice(&cur);
        cudaError_t e = cudaSetDevice(device);
        void *p = nullptr;
        if (e == cudaSuccess)
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (cur >= 0 && cur != device)
            cudaSetDevice(cur);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_na_ptr[device] = p;
    }
    *out = static_cast<uint8_t *>(g_na_ptr[device]);
    return CMD_OK;
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
    uint8_t *base = nullptr;
    int rc = noalloc_scratch(eng->device, &base);
    if (rc)
        return rc;
    cudaSetDevice(eng->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    uint32_t *synd = reinterpret_cast<uint32_t *>(base);
    uint16_t *loc = reinterpret_cast<uint16_t *>(base + NA_SYND_BYTES);
    LaunchCounter lc{&eng->launches};
    cudaError_t e;
    if ((e = launch_synd_plain(key->dev, d_cts, count, synd, s, lc)) != cudaSuccess ||
        (e = launch_bm_plain(key->dev.set, reinterpret_cast<uint16_t *>(synd), count, loc, s, lc)) != cudaSuccess ||
        (e = launch_root_plain(key->dev, loc, count, d_err, d_weight, s, lc, eng->num_sms)) != cudaSuccess)
        return cuda_fail(e, "no-alloc plain path launch");
    return CMD_OK;
}
