// The drift tier's kernel (FP32, semiglobal rescue of error-rich long reads),
// compiled on its own so its strip driver gets its own register budget.
#include "pairhmm_kernel.cuh"
#include "pairhmm_launch.h"

namespace vd {

cudaError_t launch_drift_f32(const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                             const Scalars<float>& sc, int grid, cudaStream_t stream) {
  pairhmm_drift_kernel<4><<<grid, kWarpsPerBlock * kWarp, 0, stream>>>(bv, qv, tab, sc);
  return cudaGetLastError();
}

cudaError_t occupancy_drift_f32(int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_drift_kernel<4>,
                                                       kWarpsPerBlock * kWarp, 0);
}

}  // namespace vd
