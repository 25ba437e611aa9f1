// Dispatch for the fused kernel (fused_impl.cuh): picks the instantiation for
// a single-set batch or the all-sets one for mixed batches.
#include "fused_impl.cuh"

namespace cmd {

// 227 KB opt-in per CTA on sm_100, less room for the kernel's static shared memory.
size_t smem_limit_bytes() { return 232448 - 1024; }

size_t fused_smem(int set, int wpb)
{
    return dispatch_set(set, [&]<int S>() -> size_t { return fz_smem<S>(wpb); });
}

int fused_blocks_per_sm(int single_set, int wpb, size_t smem)
{
    switch (single_set) {
    case S348864: return fused_occ_1(wpb, smem);
    case S460896: return fused_occ_2(wpb, smem);
    case S6688128: return fused_occ_4(wpb, smem);
    case S6960119: return fused_occ_8(wpb, smem);
    case S8192128: return fused_occ_16(wpb, smem);
    default: return fused_occ_31(wpb, smem);
    }
}

cudaError_t launch_fused(const FusedArgs &a, int grid, int wpb, cudaStream_t s, LaunchCounter lc)
{
    size_t smem = 0;
    if (a.single_set >= 0) {
        smem = fused_smem(a.single_set, wpb);
    } else {
        for (int st = 0; st < NSETS; st++)
            smem = smem > fused_smem(st, wpb) ? smem : fused_smem(st, wpb);
    }
    if (smem > smem_limit_bytes())
        return cudaErrorInvalidConfiguration;
    cudaError_t e;
    switch (a.single_set) {
    case S348864: e = fused_launch_1(a, grid, wpb, smem, s); break;
    case S460896: e = fused_launch_2(a, grid, wpb, smem, s); break;
    case S6688128: e = fused_launch_4(a, grid, wpb, smem, s); break;
    case S6960119: e = fused_launch_8(a, grid, wpb, smem, s); break;
    case S8192128: e = fused_launch_16(a, grid, wpb, smem, s); break;
    default: e = fused_launch_31(a, grid, wpb, smem, s); break;
    }
    if (e == cudaSuccess)
        lc.bump();
    return e;
}

}  // namespace cmd
