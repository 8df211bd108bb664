// Selects the compiled kernel instantiation for a (type, mode) pair.
#include "pairhmm_launch.h"

namespace vd {

#define VD_DECL(T, tn, mn)                                                                          \
  cudaError_t launch_##tn##_##mn(const BatchView&, const QueueView&, const Tables<T>*, const Scalars<T>&, \
                                 int, int, cudaStream_t);                                           \
  cudaError_t occupancy_##tn##_##mn(int*);
VD_DECL(float, f32, sg)
VD_DECL(float, f32, an)
VD_DECL(double, f64, sg)
VD_DECL(double, f64, an)
#undef VD_DECL

cudaError_t launch_f32(bool anchored, const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                       const Scalars<float>& sc, int tier, int grid, cudaStream_t stream) {
  return anchored ? launch_f32_an(bv, qv, tab, sc, tier, grid, stream)
                  : launch_f32_sg(bv, qv, tab, sc, tier, grid, stream);
}
cudaError_t launch_f64(bool anchored, const BatchView& bv, const QueueView& qv, const Tables<double>* tab,
                       const Scalars<double>& sc, int tier, int grid, cudaStream_t stream) {
  return anchored ? launch_f64_an(bv, qv, tab, sc, tier, grid, stream)
                  : launch_f64_sg(bv, qv, tab, sc, tier, grid, stream);
}
cudaError_t occupancy_f32(bool anchored, int* b) { return anchored ? occupancy_f32_an(b) : occupancy_f32_sg(b); }
cudaError_t occupancy_f64(bool anchored, int* b) { return anchored ? occupancy_f64_an(b) : occupancy_f64_sg(b); }

}  // namespace vd
