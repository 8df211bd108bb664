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
// two-read items (FP32, semiglobal): wide = split..8 rows per lane (12 warps per SM), else
// 1..split-1 (16 warps per SM); split is 6 or 7
cudaError_t launch_pair_f32(bool wide, int split, const BatchView& bv, const QueueView& qv,
                            const Tables<float>* tab, const Scalars<float>& sc, int grid, cudaStream_t stream);
cudaError_t occupancy_pair_f32(bool wide, int split, int* blocks_per_sm);
// the drift tier (FP32 semiglobal rescue with per-row power-of-two boosts)
cudaError_t launch_drift_f32(const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                             const Scalars<float>& sc, int grid, cudaStream_t stream);
cudaError_t occupancy_drift_f32(int* blocks_per_sm);
// long reads, a read against two haplotypes per item (pairhmm_long.cuh), R = 8 or 4 rows
// per lane; block: the CTA's warps split each strip (block per item), else warp per item
cudaError_t launch_long_f32(int R, bool block, const BatchView& bv, const QueueView& qv, const Tables<float>* tab,
                            const Scalars<float>& sc, int grid, cudaStream_t stream);
cudaError_t occupancy_long_f32(int R, bool block, int* blocks_per_sm);
// gradient kernel (pairhmm_backward.cuh), FP32 and FP64 passes
struct GradTables;
struct GradScalars;
struct GradView;
cudaError_t launch_grad_f32(const BatchView& bv, const GradView& gv, const Tables<float>* tab,
                            const Scalars<float>& sc, const GradTables* gt, const GradScalars& gs, int grid,
                            cudaStream_t stream);
cudaError_t launch_grad_f64(const BatchView& bv, const GradView& gv, const Tables<double>* tab,
                            const Scalars<double>& sc, const GradTables* gt, const GradScalars& gs, int grid,
                            cudaStream_t stream);
cudaError_t occupancy_grad(bool fp64, int* blocks_per_sm);
// bytes of one warp slot's checkpoints and segment buffer (sized for the FP64 pass)
long long grad_slot_bytes(int R, int m, bool store_all);
// region post-processing (pairhmm_genotype.cu)
cudaError_t launch_genotype_rows(const double* ln, const int64_t* row_off, const int32_t* row_h,
                                 const double* mq_error, int64_t n_reads, double* values, double* certainty,
                                 int sm_count, cudaStream_t stream);
cudaError_t launch_genotype_gl(const double* values, const int64_t* region_out_off, const int64_t* region_reads,
                               const int32_t* region_h, const int64_t* gl_off, const int64_t* acc_off,
                               int64_t n_regions, double prior, double* acc, double* gl, int sm_count,
                               cudaStream_t stream);
cudaError_t launch_genotype_ties(const double* gl, const int64_t* gl_off, const int32_t* region_h,
                                 const int64_t* region_reads, int64_t n_regions, int* flags, cudaStream_t stream);
// sets the message vd_last_error returns on this thread; returns code
int report_error(int code, const char* msg);
// model tables for (gap, ext, optional per-bin Phred offsets), built on the host
void build_model_tables(double gap, double ext, const double* offsets, Tables<float>* f32, Tables<double>* f64,
                        Scalars<float>* s32, Scalars<double>* s64);
}  // namespace vd
