// Instantiation of the fused kernel for set mask 31 (bit i = set index i).
#include "fused_impl.cuh"

namespace cmd {

cudaError_t fused_launch_31(const FusedArgs &a, int grid, int wpb, size_t smem, cudaStream_t s)
{
    return wpb == 8 ? launch_k<31, 8>(a, grid, smem, s) : launch_k<31, 4>(a, grid, smem, s);
}

int fused_occ_31(int wpb, size_t smem) { return wpb == 8 ? occupancy<31, 8>(smem) : occupancy<31, 4>(smem); }

}  // namespace cmd
