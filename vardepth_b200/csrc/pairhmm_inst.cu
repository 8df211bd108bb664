// One instantiation of the wavefront kernel, selected at compile time:
//   -DVD_FP64=0|1  arithmetic type (float: primary tier, double: rescue tiers)
//   -DVD_ANCH=0|1  semiglobal or anchored mode
// The build compiles this file four times so the instantiations compile in
// parallel; each object exports one launcher and one occupancy query.
#include "pairhmm_kernel.cuh"
#include "pairhmm_launch.h"

#if VD_FP64
#define VD_T double
#define VD_TNAME f64
#else
#define VD_T float
#define VD_TNAME f32
#endif
#if VD_ANCH
#define VD_MNAME an
#else
#define VD_MNAME sg
#endif
#define VD_CAT3(a, b, c) a##_##b##_##c
#define VD_NAME(a, b, c) VD_CAT3(a, b, c)

namespace vd {

cudaError_t VD_NAME(launch, VD_TNAME, VD_MNAME)(const BatchView& bv, const QueueView& qv,
                                                const Tables<VD_T>* tab, const Scalars<VD_T>& sc,
                                                int tier, int grid, cudaStream_t stream) {
  pairhmm_kernel<VD_T, (VD_ANCH != 0)><<<grid, kWarpsPerBlock * kWarp, 0, stream>>>(bv, qv, tab, sc, tier);
  return cudaGetLastError();
}

cudaError_t VD_NAME(occupancy, VD_TNAME, VD_MNAME)(int* blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_kernel<VD_T, (VD_ANCH != 0)>,
                                                       kWarpsPerBlock * kWarp, 0);
}

#if !VD_FP64 && !VD_ANCH
// Two tilings of the rows-per-lane range: split 6 runs 1-5 rows at 16 warps per
// SM and 6-8 at 12; split 7 moves 6 rows to the 16-warp kernel (128 registers,
// a few spills) -- the autotuner measures which is faster for a batch.
cudaError_t launch_pair_f32(bool wide, int split, const BatchView& bv, const QueueView& qv,
                            const Tables<float>* tab, const Scalars<float>& sc, int grid, cudaStream_t stream) {
  const int threads = kWarpsPerBlock * kWarp;
  if (split == 7) {
    if (wide) pairhmm_pair_kernel<7, 8, 3><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
    else pairhmm_pair_kernel<1, 6, 4><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
  } else {
    if (wide) pairhmm_pair_kernel<6, 8, 3><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
    else pairhmm_pair_kernel<1, 5, 4><<<grid, threads, 0, stream>>>(bv, qv, tab, sc);
  }
  return cudaGetLastError();
}

cudaError_t occupancy_pair_f32(bool wide, int split, int* blocks_per_sm) {
  const int threads = kWarpsPerBlock * kWarp;
  if (split == 7)
    return wide ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_pair_kernel<7, 8, 3>, threads, 0)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_pair_kernel<1, 6, 4>, threads, 0);
  return wide ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_pair_kernel<6, 8, 3>, threads, 0)
              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pairhmm_pair_kernel<1, 5, 4>, threads, 0);
}
#endif

}  // namespace vd
