// Instantiations of the long-read kernels (pairhmm_long.cuh): warp per item
// and block per item, each with 256-row strips (8 rows per lane) and 128-row
// strips (4 rows per lane).
#include "pairhmm_launch.h"
#include "pairhmm_long.cuh"

namespace vd {

cudaError_t launch_long_f32(int R, bool block, const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                            const Scalars<float>& sc, int grid, cudaStream_t stream) {
  const int threads = kWarpsPerBlock * kWarp;
  if (block) {
    if (R == 8) pairhmm_long_block_kernel<8, 3><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
    else pairhmm_long_block_kernel<4, 4><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
  } else {
    if (R == 8) pairhmm_long_kernel<8, 3><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
    else pairhmm_long_kernel<4, 4><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
  }
  return cudaGetLastError();
}

cudaError_t occupancy_long_f32(int R, bool block, int* blocks_per_sm) {
  const int threads = kWarpsPerBlock * kWarp;
  if (block)
    return R == 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_long_block_kernel<8, 3>, threads, 0)
                  : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_long_block_kernel<4, 4>, threads, 0);
  return R == 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_long_kernel<8, 3>, threads, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_long_kernel<4, 4>, threads, 0);
}

}  // namespace vd
