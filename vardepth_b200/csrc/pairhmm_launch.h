// Host-side launchers of the instantiated kernels.
#pragma once
#include <cuda_runtime.h>
#include "pairhmm_core.cuh"

namespace vd {
cudaError_t launch_f32(bool anchored, const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                       const Scalars<float>& sc, int tier, int grid, cudaStream_t stream);
cudaError_t launch_f64(bool anchored, const BatchView& bv, const QueueView& qv, const Tables<double>* tab,
                       const Scalars<double>& sc, int tier, int grid, cudaStream_t stream);
cudaError_t occupancy_f32(bool anchored, int* blocks_per_sm);
cudaError_t occupancy_f64(bool anchored, int* blocks_per_sm);
// two-read items (FP32, semiglobal)
cudaError_t launch_pair_f32(const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                            const Scalars<float>& sc, int grid, cudaStream_t stream);
cudaError_t occupancy_pair_f32(int* blocks_per_sm);
}  // namespace vd
