// Instantiations and launchers of the reverse-wavefront gradient kernel
// (pairhmm_backward.cuh): an FP32 pass and an FP64 pass for the pairs whose
// FP32 forward underflowed.
#include "pairhmm_backward.cuh"
#include "pairhmm_launch.h"

namespace vd {

namespace {
template <typename T>
constexpr int dyn_smem() { return kWarpsPerBlock * grad_smem_per_warp<T>(); }

// the sub-segment buffers exceed the 48 KB default of dynamic shared memory
template <typename T>
cudaError_t allow_smem() {
  cudaError_t e = cudaFuncSetAttribute(pairhmm_grad_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       dyn_smem<T>());
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(pairhmm_grad_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              dyn_smem<T>());
}
}  // namespace

cudaError_t launch_grad_f32(const BatchView& bv, const GradView& gv, const Tables<float>* tab,
                            const Scalars<float>& sc, const GradTables* gt, const GradScalars& gs, int grid,
                            cudaStream_t stream) {
  cudaError_t e = allow_smem<float>();
  if (e != cudaSuccess) return e;
  if (gv.anchored)
    pairhmm_grad_kernel<float, true><<<grid, kWarpsPerBlock * kWarp, dyn_smem<float>(), stream>>>(bv, gv, tab, sc, gt,
                                                                                                  gs);
  else
    pairhmm_grad_kernel<float, false><<<grid, kWarpsPerBlock * kWarp, dyn_smem<float>(), stream>>>(bv, gv, tab, sc,
                                                                                                   gt, gs);
  return cudaGetLastError();
}

cudaError_t launch_grad_f64(const BatchView& bv, const GradView& gv, const Tables<double>* tab,
                            const Scalars<double>& sc, const GradTables* gt, const GradScalars& gs, int grid,
                            cudaStream_t stream) {
  cudaError_t e = allow_smem<double>();
  if (e != cudaSuccess) return e;
  if (gv.anchored)
    pairhmm_grad_kernel<double, true><<<grid, kWarpsPerBlock * kWarp, dyn_smem<double>(), stream>>>(bv, gv, tab, sc,
                                                                                                    gt, gs);
  else
    pairhmm_grad_kernel<double, false><<<grid, kWarpsPerBlock * kWarp, dyn_smem<double>(), stream>>>(bv, gv, tab, sc,
                                                                                                     gt, gs);
  return cudaGetLastError();
}

cudaError_t occupancy_grad(bool fp64, int* blocks_per_sm) {
  cudaError_t e = fp64 ? allow_smem<double>() : allow_smem<float>();
  if (e != cudaSuccess) return e;
  return fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_grad_kernel<double, false>,
                                                              kWarpsPerBlock * kWarp, dyn_smem<double>())
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_grad_kernel<float, false>,
                                                              kWarpsPerBlock * kWarp, dyn_smem<float>());
}

long long grad_slot_bytes(int R, int m, bool store_all) {
  return grad_slot_elems(R, m, store_all) * (long long)sizeof(double);
}

}  // namespace vd
