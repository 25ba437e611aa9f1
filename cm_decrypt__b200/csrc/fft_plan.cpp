// Host-side plans of the additive FFT (Gao-Mateer) that the fused kernel uses
// to evaluate an error locator at every element of GF(2^m).
//
// The reference evaluates the locator at each support point by Horner
// (root_13.c:216-240).  Here the locator f (degree <= t < 2^D) is evaluated
// at all 2^m field elements at once, and the key's support network then moves
// the zero flags to support order (see the fused kernel).  The recursion, on
// an m-element basis B = (B_1..B_k):
//   g(x) = f(B_1 x);  g = g0(x^2+x) + x g1(x^2+x)   (Taylor expansion)
//   evaluate g0, g1 on the basis (G_i^2 + G_i), G_i = B_i / B_1, i >= 2;
//   f(B_1 a) = g0(a^2+a) + a g1(a^2+a),  f(B_1 (a+1)) = f(B_1 a) + g1(a^2+a).
// With B_{j+1} = x^j the top-level output index q is the integer value of
// the evaluation point; the kernel keeps output q at position bitrev_m(q), so
// every butterfly pairs whole 32-bit words of the bitsliced array.
//
// The same recursion, transposed, gives the serving path's syndromes: the
// power sums sum_a u_a a^j (j < 2t) of values u_a at all 2^m elements (see
// latency.cu).  That needs 2t coefficients, depth D' with 2^D' >= 2t, one
// level more than the root search for t = 96 and 119; the tables below go to
// depth D' (the root search reads the first D levels, whose entries do not
// depend on how deep the tables go).
//
// Per depth d < D' this file computes
//   * scalpow[d][i] = b_d^i (i < 2^(D'-d)), b_d the first basis element at
//     depth d -- the scaling g(x) = f(b_d x) of the radix conversion;
//   * the twiddles: the butterfly of depth d pairs positions Y and
//     Y + 2^(m-d-1); its multiplier a(Y) depends on r = Y mod 2^(m-d-1):
//     a = sum_j bit(m-d-2-j of r) * G_{j+2}, stored bitsliced, 32 values r
//     per word, m planes padded to 16.
#include <cstring>
#include <vector>

#include "engine.h"

namespace cmd {
namespace {

uint32_t fmul(uint32_t a, uint32_t b, int m)
{
    const uint32_t poly = m == 13 ? 0x201Bu : 0x1009u;
    uint32_t p = 0;
    for (int i = 0; i < m; i++)
        if ((b >> i) & 1u)
            p ^= a << i;
    for (int i = 2 * m - 2; i >= m; i--)
        if ((p >> i) & 1u)
            p ^= poly << (i - m);
    return p;
}

uint32_t finv(uint32_t a, int m)
{
    uint32_t r = 1, x = a;
    for (uint32_t e = (1u << m) - 2; e; e >>= 1) {
        if (e & 1u)
            r = fmul(r, x, m);
        x = fmul(x, x, m);
    }
    return r;
}

struct FftPlanHost {
    int D = 0;
    std::vector<uint16_t> scalpow;  // [8][256]
    std::vector<uint32_t> tw;       // [words][16]
};

FftPlanHost make_fft_plan(int set)
{
    const SetInfo si = set_info(set);
    const int m = si.m;
    FftPlanHost p;
    p.D = synd_depth(si.t);
    p.scalpow.assign(8 * 256, 0);
    std::vector<uint32_t> B(m);
    for (int j = 0; j < m; j++)
        B[j] = 1u << j;
    for (int d = 0; d < p.D; d++) {
        const uint32_t b1 = B[0];
        uint32_t pw = 1;
        for (int i = 0; i < (1 << (p.D - d)); i++) {
            p.scalpow[d * 256 + i] = (uint16_t)pw;
            pw = fmul(pw, b1, m);
        }
        const uint32_t inv = finv(b1, m);
        std::vector<uint32_t> G(B.size());
        for (size_t i = 0; i < B.size(); i++)
            G[i] = fmul(B[i], inv, m);
        const int nbits = m - d - 1;
        const int words = 1 << (nbits - 5);
        const size_t base = p.tw.size();
        p.tw.resize(base + (size_t)words * 16, 0);
        for (int r = 0; r < (1 << nbits); r++) {
            uint32_t a = 0;
            for (int j = 0; j < nbits; j++)
                if ((r >> (nbits - 1 - j)) & 1)
                    a ^= G[j + 1];
            for (int k = 0; k < m; k++)
                p.tw[base + (size_t)(r >> 5) * 16 + k] |= ((a >> k) & 1u) << (r & 31);
        }
        std::vector<uint32_t> nb(B.size() - 1);
        for (size_t i = 1; i < B.size(); i++)
            nb[i - 1] = fmul(G[i], G[i], m) ^ G[i];
        B.swap(nb);
    }
    return p;
}

size_t al256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

int upload_fft_plans(cmd_engine *eng)
{
    FftPlanHost plans[NSETS];
    size_t off[NSETS][2], total = 0;
    for (int s = 0; s < NSETS; s++) {
        plans[s] = make_fft_plan(s);
        off[s][0] = total;
        total = al256(total + plans[s].scalpow.size() * 2);
        off[s][1] = total;
        total = al256(total + plans[s].tw.size() * 4);
    }
    if (!budget_take(eng, total)) {
        set_last_error("root-search tables exceed the engine HBM budget");
        return CMD_E_BUDGET;
    }
    std::vector<uint8_t> host(total, 0);
    for (int s = 0; s < NSETS; s++) {
        memcpy(host.data() + off[s][0], plans[s].scalpow.data(), plans[s].scalpow.size() * 2);
        memcpy(host.data() + off[s][1], plans[s].tw.data(), plans[s].tw.size() * 4);
    }
    void *mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, total);
    if (e == cudaSuccess)
        e = cudaMemcpy(mem, host.data(), total, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (mem)
            cudaFree(mem);
        budget_give(eng, total);
        return cuda_fail(e, "root-search tables");
    }
    eng->fft_mem = mem;
    eng->fft_bytes = total;
    for (int s = 0; s < NSETS; s++) {
        eng->fft[s].scalpow = reinterpret_cast<const uint16_t *>(static_cast<uint8_t *>(mem) + off[s][0]);
        eng->fft[s].tw = reinterpret_cast<const uint32_t *>(static_cast<uint8_t *>(mem) + off[s][1]);
    }
    return CMD_OK;
}

void release_fft_plans(cmd_engine *eng)
{
    if (eng->fft_mem) {
        cudaFree(eng->fft_mem);
        budget_give(eng, eng->fft_bytes);
        eng->fft_mem = nullptr;
        eng->fft_bytes = 0;
    }
}

}  // namespace cmd
