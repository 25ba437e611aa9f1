// Instantiation of the fused kernel for set mask 2 (bit i = set index i).
#include "fused_impl.cuh"

namespace cmd {

cudaError_t fused_launch_2(const FusedArgs &a, int grid, int wpb, size_t smem, cudaStream_t s)
{
    return wpb == 8 ? launch_k<2, 8>(a, grid, smem, s) : launch_k<2, 4>(a, grid, smem, s);
}

int fused_occ_2(int wpb, size_t smem) { return wpb == 8 ? occupancy<2, 8>(smem) : occupancy<2, 4>(smem); }

}  // namespace cmd
