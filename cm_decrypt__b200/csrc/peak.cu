// Integer-ALU roofline denominator: sustained LOP3 (3-input logic op) issue
// rate of the whole GPU, the instruction the bitsliced GF(2^m) kernels are
// made of.  Each thread runs 16 independent dependency chains of lop3.b32 so
// latency is hidden and the ALU pipe is the only limit.
#include <cuda_runtime.h>

#include "engine.h"

namespace cmd {

constexpr int PEAK_CHAINS = 16, PEAK_ITERS = 2048;

__global__ void __launch_bounds__(256) k_lop3_peak(uint32_t seed, uint32_t *out)
{
    uint32_t r[PEAK_CHAINS];
#pragma unroll
    for (int i = 0; i < PEAK_CHAINS; i++)
        r[i] = seed * (threadIdx.x + 1) + i * 0x9E3779B9u + blockIdx.x;
#pragma unroll 1
    for (int it = 0; it < PEAK_ITERS; it++) {
#pragma unroll
        for (int i = 0; i < PEAK_CHAINS; i++) {
            uint32_t o;
            asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(o)
                         : "r"(r[i]), "r"(r[(i + 1) % PEAK_CHAINS]), "r"(r[(i + 5) % PEAK_CHAINS]));
            r[i] = o;
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < PEAK_CHAINS; i++)
        x ^= r[i];
    if (x == 0x12345678u)  // practically never; keeps the chains live
        out[0] = x;
}

}  // namespace cmd

using namespace cmd;

// Measures LOP3 lane-operations per second on the engine's device.
extern "C" int cmd_bench_int_peak(cmd_engine *eng, double *lop3_lane_ops_per_s)
{
    if (!eng || !lop3_lane_ops_per_s)
        return CMD_E_ARG;
    cudaSetDevice(eng->device);
    std::lock_guard<std::mutex> lk(eng->mu);
    uint32_t *d_out = nullptr;
    cudaEvent_t e0, e1;
    cudaError_t e = cudaMalloc(&d_out, 64);
    if (e != cudaSuccess)
        return cuda_fail(e, "cudaMalloc(peak)");
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = eng->num_sms * 8, threads = 256;
    double best = 0;
    for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {
        cudaEventRecord(e0, eng->stream);
        k_lop3_peak<<<blocks, threads, 0, eng->stream>>>(rep + 1, d_out);
        eng->launches.fetch_add(1);
        cudaEventRecord(e1, eng->stream);
        e = cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = (double)blocks * threads * PEAK_ITERS * PEAK_CHAINS;
        if (rep > 0 && ms > 0)
            best = std::max(best, ops / (ms * 1e-3));
    }
    if (e == cudaSuccess)
        e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d_out);
    if (e != cudaSuccess)
        return cuda_fail(e, "lop3 peak kernel");
    *lop3_lane_ops_per_s = best;
    return CMD_OK;
}
