// KEM decapsulation around the decrypt path.  No counterpart in the
// reference, which encapsulates only: kem/common/core/operations.c:15-34
// computes C = [I | T] e and K = SHAKE256(1 || e || C) (32 bytes).  The
// Classic McEliece decapsulation inverts that with implicit rejection:
//
//   e = decrypt(C)                       (the engine's fused kernel)
//   accept = padding bits mt..8*ct-1 of C are zero  &&  wt(e) == t
//            &&  C == [I | T] e          (e re-encodes to C)
//   K = SHAKE256(b || v || C),  b = accept,  v = accept ? e : s
//
// with T the systematic public key (derived once per key on the device from
// the key's support and Goppa polynomial by the key generation's elimination)
// and s the random string stored at the end of the secret key.
//
// k_decap: 8 warps per CTA, lane = ciphertext, 256 ciphertexts per CTA.
//  1. re-encoding: each lane keeps the mt-bit word vector acc = T * e[mt..n)
//     in registers; the columns of T stream through shared memory in
//     32-column chunks (cp.async double buffer shared by the CTA) and every
//     column is masked by the lane's error bit -- every column for every
//     ciphertext, so the work and the memory traffic do not depend on e;
//  2. acc ^ e[0..mt) ^ C must vanish; padding and weight checks;
//  3. SHAKE256 of the 1 + n/8 + ct byte preimage, one lane per ciphertext
//     (Keccak-f[1600] as defined in FIPS 202; round constants and rotation
//     offsets derived from the standard's definitions at compile time); the
//     preimage's v bytes are selected with masks.
#include <cstring>
#include <mutex>

#include "engine.h"
#include "fused_impl.cuh"
#include "keccak.cuh"

namespace cmd {

namespace {

constexpr int COLS = 32;  // public-key columns per staged chunk

template <int S> struct DecapDims {
    using P = Set<S>;
    static constexpr int MT = P::M * P::T;
    static constexpr int CW = (MT + 31) / 32;        // u32 words per column
    static constexpr int CWP = (CW + 3) / 4 * 4;     // column stride (16-byte rows)
    static constexpr int XC = P::N - MT;             // columns of T
    static constexpr int NB = P::N / 8;              // bytes of e and of s
    static constexpr int MSG = 1 + NB + P::CT;       // preimage bytes
};

}  // namespace

struct DecapArgs {
    const uint8_t *cts;
    const uint32_t *err;       // error rows, nw words each
    const uint16_t *weight;
    const uint32_t *pkT;       // column c of T at pkT + c * CWP
    const uint8_t *s;          // the secret key's n/8-byte string s
    uint8_t *keys;             // 32 bytes per ciphertext
    uint8_t *accept;           // or null: 1 byte per ciphertext
    uint64_t count;
};

template <int S> __global__ void __launch_bounds__(256) k_decap(DecapArgs a)
{
    using P = Set<S>;
    using Q = DecapDims<S>;
    constexpr int CW = Q::CW, CWP = Q::CWP, XC = Q::XC, MT = Q::MT, NW = P::NW;
    extern __shared__ __align__(16) uint32_t colbuf[];  // 2 x COLS x CWP words
    const int tid = threadIdx.x, lane = tid & 31;
    const uint64_t c = (uint64_t)blockIdx.x * 256 + tid;
    const bool live = c < a.count;
    const uint64_t cc = live ? c : 0;
    const uint32_t *erow = a.err + cc * NW;

    // ---- 1. acc = T * e[mt..n), every column masked by the error bit ------
    uint32_t acc[CW];
#pragma unroll
    for (int w = 0; w < CW; w++)
        acc[w] = 0;
    constexpr int NCH = (XC + COLS - 1) / COLS;
    constexpr int CHUNK_V = COLS * CWP / 4;
    auto stage = [&](int ch) {
        uint32_t *dst = colbuf + (ch & 1) * COLS * CWP;
        const int cols = XC - ch * COLS < COLS ? XC - ch * COLS : COLS;
        for (int v = tid; v < CHUNK_V; v += 256) {
            if (v * 4 < cols * CWP)
                cp_async16(dst + 4 * v, a.pkT + (size_t)ch * COLS * CWP + 4 * v);
        }
        cp_async_commit();
    };
    stage(0);
    uint32_t ew = 0;
#pragma unroll 1
    for (int ch = 0; ch < NCH; ch++) {
        if (ch + 1 < NCH) {
            stage(ch + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const uint32_t *buf = colbuf + (ch & 1) * COLS * CWP;
        const int cols = XC - ch * COLS < COLS ? XC - ch * COLS : COLS;
#pragma unroll 1
        for (int j = 0; j < cols; j++) {
            const int bit = MT + ch * COLS + j;
            if (j == 0 || (bit & 31) == 0)
                ew = live ? erow[bit >> 5] : 0u;
            const uint32_t m = 0u - ((ew >> (bit & 31)) & 1u);
            const uint4 *col = reinterpret_cast<const uint4 *>(buf + j * CWP);
#pragma unroll
            for (int v = 0; v < CWP / 4; v++) {
                const uint4 x = col[v];
                if (4 * v + 0 < CW) acc[4 * v + 0] ^= x.x & m;
                if (4 * v + 1 < CW) acc[4 * v + 1] ^= x.y & m;
                if (4 * v + 2 < CW) acc[4 * v + 2] ^= x.z & m;
                if (4 * v + 3 < CW) acc[4 * v + 3] ^= x.w & m;
            }
        }
        __syncthreads();
    }
    if (!live)
        return;  // no block-wide barrier follows

    // ---- 2. acceptance ------------------------------------------------------
    const uint8_t *ct = a.cts + cc * P::CT;
    uint32_t diff = 0;
#pragma unroll
    for (int w = 0; w < CW; w++) {
        uint32_t cw = 0;
#pragma unroll
        for (int b = 0; b < 4; b++)
            if (4 * w + b < P::CT)
                cw |= (uint32_t)ct[4 * w + b] << (8 * b);
        uint32_t d = acc[w] ^ erow[w] ^ cw;
        if (32 * w + 32 > MT)
            d &= (1u << (MT - 32 * w)) - 1u;  // bits mt.. are the padding check's
        diff |= d;
    }
    uint32_t pad = 0;
    for (int b = MT; b < 8 * P::CT; b++)
        pad |= (ct[b >> 3] >> (b & 7)) & 1u;
    const bool ok = diff == 0 && pad == 0 && a.weight[cc] == P::T;
    const uint32_t okm = ok ? 0xFFu : 0u;
    if (a.accept)
        a.accept[cc] = ok ? 1 : 0;

    // ---- 3. K = SHAKE256(b || v || C), 32 bytes ------------------------------
    // preimage byte i: 0 -> b; 1..NB -> v; then C; then the pad10*1 padding
    // with the SHAKE domain bits (0x1F ... 0x80) over whole 136-byte blocks.
    constexpr int RATE = 136;
    constexpr int NBLK = Q::MSG / RATE + 1;
    const uint8_t *eb = reinterpret_cast<const uint8_t *>(erow);
    auto msg = [&](int i) -> uint32_t {
        if (i == 0)
            return okm & 1u;
        if (i <= Q::NB)
            return (eb[i - 1] & okm) | (a.s[i - 1] & ~okm & 0xFFu);
        if (i < Q::MSG)
            return ct[i - 1 - Q::NB];
        uint32_t v = i == Q::MSG ? 0x1Fu : 0u;
        if (i == NBLK * RATE - 1)
            v |= 0x80u;
        return v;
    };
    uint64_t A[25];
#pragma unroll
    for (int i = 0; i < 25; i++)
        A[i] = 0;
#pragma unroll 1
    for (int blk = 0; blk < NBLK; blk++) {
#pragma unroll
        for (int l = 0; l < RATE / 8; l++) {  // static lane index: A stays in registers
            uint64_t v = 0;
#pragma unroll
            for (int b = 0; b < 8; b++)
                v |= (uint64_t)msg(blk * RATE + 8 * l + b) << (8 * b);
            A[l] ^= v;
        }
        keccak_f(A);
    }
    uint64_t *out = reinterpret_cast<uint64_t *>(a.keys + cc * 32);
#pragma unroll
    for (int i = 0; i < 4; i++)
        out[i] = A[i];
    (void)lane;
}

size_t decap_pk_words(int set)
{
    return dispatch_set(set, [&]<int S>() -> size_t { return (size_t)DecapDims<S>::XC * DecapDims<S>::CWP; });
}

cudaError_t launch_decap(int set, const uint8_t *d_cts, const uint32_t *d_err, const uint16_t *d_w,
                         const uint32_t *d_pk, const uint8_t *d_s, uint8_t *d_keys, uint8_t *d_accept, size_t count,
                         cudaStream_t s, LaunchCounter lc)
{
    if (count == 0)
        return cudaSuccess;
    DecapArgs a{d_cts, d_err, d_w, d_pk, d_s, d_keys, d_accept, count};
    return dispatch_set(set, [&]<int S>() -> cudaError_t {
        const size_t smem = 2 * (size_t)COLS * DecapDims<S>::CWP * 4;  // <= 13.3 KB: no opt-in needed
        static_assert(2 * COLS * DecapDims<S>::CWP * 4 <= 48 * 1024, "decap staging");
        k_decap<S><<<(unsigned)((count + 255) / 256), 256, smem, s>>>(a);
        lc.bump();
        return cudaGetLastError();
    });
}

}  // namespace cmd

using namespace cmd;

extern "C" {

int cmd_key_prepare_decap(cmd_engine *eng, cmd_key *key)
{
    if (!eng || !key || key->eng != eng)
        return CMD_E_ARG;
    // one preparation at a time per key, so that two first calls for a key
    // derive its columns once (keys of other engines and devices prepare in
    // parallel); taken before eng->mu, which kg_pubkey_columns takes
    std::lock_guard<std::mutex> lk(key->prep_mu);
    if (key->pk)
        return CMD_OK;
    const int set = key->dev.set;
    const size_t bytes = decap_pk_words(set) * 4;
    const int cwp = dispatch_set(set, [&]<int S>() { return DecapDims<S>::CWP; });
    if (!budget_take(eng, bytes)) {
        set_last_error("public key does not fit the engine HBM budget");
        return CMD_E_BUDGET;
    }
    cudaSetDevice(eng->device);
    void *p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        budget_give(eng, bytes);
        return cuda_fail(e, "public key columns");
    }
    // the key's parity-check matrix from its device support and Goppa
    // polynomial, reduced on the device
    const int rc = kg_pubkey_columns(eng, set, key->dev.L, key->dev.g, static_cast<uint32_t *>(p), cwp);
    if (rc) {
        cudaFree(p);
        budget_give(eng, bytes);
        return rc;
    }
    key->pk = static_cast<uint32_t *>(p);
    key->pk_bytes = bytes;
    return CMD_OK;
}

int cmd_kem_decap_device(cmd_engine *eng, cmd_key *key, const uint8_t *d_cts, size_t count, uint8_t *d_keys,
                         uint8_t *d_accept, void *stream)
{
    if (!eng || !key || key->eng != eng || (count && (!d_cts || !d_keys)))
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    int rc = cmd_key_prepare_decap(eng, key);
    if (rc)
        return rc;
    const SetInfo si = set_info(key->dev.set);
    cudaSetDevice(eng->device);
    std::lock_guard<std::mutex> lk(eng->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : eng->stream;
    const size_t words = count * si.nw;
    if ((rc = eng->scratch.reserve(eng, words * 4 + count * 2 + 256)))
        return rc;
    uint32_t *d_err = static_cast<uint32_t *>(eng->scratch.ptr);
    uint16_t *d_w = reinterpret_cast<uint16_t *>(d_err + words);
    if ((rc = run_fused_single(eng, key, d_cts, count, d_err, d_w, s)))
        return rc;
    const uint8_t *d_s = key->dev.sk + 40 + 2 * si.t + si.cond;
    cudaError_t e = launch_decap(key->dev.set, d_cts, d_err, d_w, key->pk, d_s, d_keys, d_accept, count, s,
                                 LaunchCounter{&eng->launches});
    return e == cudaSuccess ? CMD_OK : cuda_fail(e, "decapsulation kernel");
}

int cmd_kem_decap(cmd_engine *eng, cmd_key *key, const uint8_t *h_cts, size_t count, uint8_t *h_keys,
                  uint8_t *h_accept)
{
    if (!eng || !key || key->eng != eng || (count && (!h_cts || !h_keys)))
        return CMD_E_ARG;
    if (count == 0)
        return CMD_OK;
    int rc = cmd_key_prepare_decap(eng, key);
    if (rc)
        return rc;
    const SetInfo si = set_info(key->dev.set);
    cudaSetDevice(eng->device);
    const size_t chunk = std::min<size_t>(count, (size_t)1 << 20);
    uint8_t *d_cts = nullptr, *d_keys = nullptr, *d_acc = nullptr;
    {
        std::lock_guard<std::mutex> lk(eng->mu);
        if ((rc = eng->io.reserve(eng, chunk * (si.ct + 32 + 1) + 1024)))
            return rc;
        uint8_t *base = static_cast<uint8_t *>(eng->io.ptr);
        d_cts = base;
        d_keys = base + (chunk * si.ct + 255) / 256 * 256;
        d_acc = d_keys + chunk * 32;
    }
    cudaStream_t s = eng->stream;
    for (size_t c0 = 0; c0 < count; c0 += chunk) {
        const size_t n = std::min(chunk, count - c0);
        cudaError_t e = cudaMemcpyAsync(d_cts, h_cts + c0 * si.ct, n * si.ct, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess)
            return cuda_fail(e, "cudaMemcpyAsync(cts H2D)");
        if ((rc = cmd_kem_decap_device(eng, key, d_cts, n, d_keys, d_acc, s)))
            return rc;
        e = cudaMemcpyAsync(h_keys + c0 * 32, d_keys, n * 32, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && h_accept)
            e = cudaMemcpyAsync(h_accept + c0, d_acc, n, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(s);
        if (e != cudaSuccess)
            return cuda_fail(e, "decapsulation D2H");
    }
    return CMD_OK;
}

}  // extern "C"
