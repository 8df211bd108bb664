// Instantiations of the long-read kernel (pairhmm_long.cuh): 256-row strips
// (8 rows per lane) and 128-row strips (4 rows per lane).
#include "pairhmm_launch.h"
#include "pairhmm_long.cuh"

namespace vd {

cudaError_t launch_long_f32(int R, const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                            const Scalars<float>& sc, int grid, cudaStream_t stream) {
  if (R == 8) pairhmm_long_kernel<8, 3><<<grid, kWarpsPerBlock * kWarp, 0, stream>>>(bv, qv, tab, sc);
  else pairhmm_long_kernel<4, 4><<<grid, kWarpsPerBlock * kWarp, 0, stream>>>(bv, qv, tab, sc);
  return cudaGetLastError();
}

cudaError_t occupancy_long_f32(int R, int* blocks_per_sm) {
  return R == 8 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_long_kernel<8, 3>,
                                                                kWarpsPerBlock * kWarp, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_long_kernel<4, 4>,
                                                                kWarpsPerBlock * kWarp, 0);
}

}  // namespace vd
