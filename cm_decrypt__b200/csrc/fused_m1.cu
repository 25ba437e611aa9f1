// Instantiation of the fused kernel for set mask 1 (bit i = set index i).
#include "fused_impl.cuh"

namespace cmd {

cudaError_t fused_launch_1(const FusedArgs &a, int grid, int wpb, size_t smem, cudaStream_t s)
{
    return wpb == 8 ? launch_k<1, 8>(a, grid, smem, s) : launch_k<1, 4>(a, grid, smem, s);
}

int fused_occ_1(int wpb, size_t smem) { return wpb == 8 ? occupancy<1, 8>(smem) : occupancy<1, 4>(smem); }

}  // namespace cmd
