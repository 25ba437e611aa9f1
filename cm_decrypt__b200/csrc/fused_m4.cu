// Instantiation of the fused kernel for set mask 4 (bit i = set index i).
#include "fused_impl.cuh"

namespace cmd {

cudaError_t fused_launch_4(const FusedArgs &a, int grid, int wpb, size_t smem, cudaStream_t s)
{
    return wpb == 8 ? launch_k<4, 8>(a, grid, smem, s) : launch_k<4, 4>(a, grid, smem, s);
}

int fused_occ_4(int wpb, size_t smem) { return wpb == 8 ? occupancy<4, 8>(smem) : occupancy<4, 4>(smem); }

}  // namespace cmd
