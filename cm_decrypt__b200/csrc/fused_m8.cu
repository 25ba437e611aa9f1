// Instantiation of the fused kernel for set mask 8 (bit i = set index i).
#include "fused_impl.cuh"

namespace cmd {

cudaError_t fused_launch_8(const FusedArgs &a, int grid, int wpb, size_t smem, cudaStream_t s)
{
    return wpb == 8 ? launch_k<8, 8>(a, grid, smem, s) : launch_k<8, 4>(a, grid, smem, s);
}

int fused_occ_8(int wpb, size_t smem) { return wpb == 8 ? occupancy<8, 8>(smem) : occupancy<8, 4>(smem); }

}  // namespace cmd
