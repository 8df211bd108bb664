// Instantiations and launchers of the reverse-wavefront gradient kernel
// (pairhmm_backward.cuh): an FP32 pass and an FP64 pass for the pairs whose
// FP32 forward underflowed.
#include "pairhmm_backward.cuh"
#include "pairhmm_launch.h"

namespace vd {

cudaError_t launch_grad_f32(const BatchView& bv, const GradView& gv, const Tables<float>* tab,
                            const Scalars<float>& sc, const GradTables* gt, const GradScalars& gs, int grid,
                            cudaStream_t stream) {
  pairhmm_grad_kernel<float><<<grid, kWarpsPerBlock * kWarp, 0, stream>>>(bv, gv, tab, sc, gt, gs);
  return cudaGetLastError();
}

cudaError_t launch_grad_f64(const BatchView& bv, const GradView& gv, const Tables<double>* tab,
                            const Scalars<double>& sc, const GradTables* gt, const GradScalars& gs, int grid,
                            cudaStream_t stream) {
  pairhmm_grad_kernel<double><<<grid, kWarpsPerBlock * kWarp, 0, stream>>>(bv, gv, tab, sc, gt, gs);
  return cudaGetLastError();
}

cudaError_t occupancy_grad(bool fp64, int* blocks_per_sm) {
  return fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_grad_kernel<double>,
                                                              kWarpsPerBlock * kWarp, 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_grad_kernel<float>,
                                                              kWarpsPerBlock * kWarp, 0);
}

long long grad_slot_bytes(int R, int m, bool store_all) {
  return grad_slot_elems(R, m, store_all) * (long long)sizeof(double);
}

}  // namespace vd
