// Region post-processing on the device, fused after the forward pass: the
// likelihood rows of each read are normalised as caller/native/caller/
// molecule_rows.py:6-14 (normalized_rows) does, and every region's unordered
// diploid genotype log-likelihoods are summed over its reads in VCF order as
// caller/native/caller/triangular.py:13-24 does without an artifact prior
// ((L_a + L_b) / 2) and caller/native/caller/mixture_general.cpp:9-37 does
// with one (allele-balance and contamination mixtures).  FP64 throughout, as
// the reference's numpy and C++.
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "pairhmm_launch.h"

namespace vd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
__constant__ double c_balance[7] = {.2, .3, .4, .5, .6, .7, .8};
__constant__ double c_balance_w[7] = {.025, .1, .225, .3, .225, .1, .025};
__constant__ double c_theta[4] = {.02, .1, .2, .3};
__constant__ double c_theta_w[4] = {.4, .35, .2, .05};

__device__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// log(exp(x) + exp(y)) with the exact doubling of equal arguments
__device__ double log_add(double x, double y) {
  if (x == y) return x + 0.6931471805599453094;
  return fmax(x, y) + log1p(exp(-fabs(x - y)));
}

// One warp per read: v = exp(ll - max ll), v' = (1 - e_mq) v + e_mq mean(v),
// certainty = max ln v' - min ln v' (ln floored at 1e-300).
__global__ void rows_kernel(const double* __restrict__ ln, const int64_t* __restrict__ row_off,
                            const int32_t* __restrict__ row_h, const double* __restrict__ mq_error,
                            int64_t n_reads, double* __restrict__ values, double* __restrict__ certainty) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < n_reads; r += warps) {
    const int H = row_h[r];
    const double* l = ln + row_off[r];
    double* v = values + row_off[r];
    if (H <= 0) {
      if (lane == 0) certainty[r] = __longlong_as_double(0x7ff8000000000000LL);
      continue;
    }
    double mx = -HUGE_VAL;
    for (int h = lane; h < H; h += 32) mx = fmax(mx, l[h]);
    mx = warp_max(mx);
    double sum = 0.0;
    for (int h = lane; h < H; h += 32) sum += exp(l[h] - mx);
    const double mean = warp_sum(sum) / (double)H;
    const double e = mq_error[r];
    double hi = -HUGE_VAL, lo = HUGE_VAL;
    bool nan = false;
    for (int h = lane; h < H; h += 32) {
      const double x = (1.0 - e) * exp(l[h] - mx) + e * mean;
      v[h] = x;
      const double lx = log(fmax(1e-300, x));
      nan |= x != x;
      hi = fmax(hi, lx);
      lo = fmin(lo, lx);
    }
    hi = warp_max(hi);
    lo = warp_min(lo);
    nan = __any_sync(kFull, nan);
    if (lane == 0) certainty[r] = nan ? __longlong_as_double(0x7ff8000000000000LL) : hi - lo;
  }
}

// One block per region: accumulator (pair, mixture component) sums ln over
// the region's rows, then each pair combines its components.
__global__ void gl_kernel(const double* __restrict__ values, const int64_t* __restrict__ region_out_off,
                          const int64_t* __restrict__ region_reads, const int32_t* __restrict__ region_h,
                          const int64_t* __restrict__ gl_off, const int64_t* __restrict__ acc_off,
                          int64_t n_regions, double prior, double* __restrict__ acc, double* __restrict__ gl) {
  for (int64_t g = blockIdx.x; g < n_regions; g += gridDim.x) {
    const int H = region_h[g];
    const int64_t R = region_reads[g];
    if (H <= 0) continue;
    const double* v = values + region_out_off[g];
    const int P = H * (H + 1) / 2;
    const int M = prior < 0.0 ? 1 : 7 + (prior > 0.0 ? 4 * H : 0);
    double* a = acc + acc_off[g];
    for (int idx = threadIdx.x; idx < P * M; idx += blockDim.x) {
      const int p = idx / M, j = idx - p * M;
      int b = (int)((sqrt(8.0 * p + 1.0) - 1.0) * 0.5);
      while (b * (b + 1) / 2 > p) --b;
      while ((b + 1) * (b + 2) / 2 <= p) ++b;
      const int ia = p - b * (b + 1) / 2, ib = b;
      double s = 0.0;
      if (prior < 0.0) {
        // numpy's maximum (triangular.py:16) keeps a NaN row (an empty read) as NaN
        for (int64_t r = 0; r < R; ++r) {
          const double t = (v[r * H + ia] + v[r * H + ib]) / 2;
          s += log(t != t ? t : fmax(1e-300, t));
        }
      } else if (j < 7) {
        // std::max(1e-300, x) of mixture_general.cpp:22-24 turns NaN into 1e-300 (fmax does too)
        const double w = c_balance[j];
        for (int64_t r = 0; r < R; ++r) s += log(fmax(1e-300, w * v[r * H + ia] + (1 - w) * v[r * H + ib]));
      } else {
        const int jj = (j - 7) / H, c = (j - 7) - jj * H;
        const double t = c_theta[jj];
        for (int64_t r = 0; r < R; ++r)
          s += log(fmax(1e-300, (1 - t) * (v[r * H + ia] + v[r * H + ib]) / 2 + t * v[r * H + c]));
      }
      a[idx] = s;
    }
    __syncthreads();
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
      const double* t = a + (int64_t)p * M;
      double out;
      if (prior < 0.0) {
        out = t[0];
      } else {
        double clean = t[0] + log(c_balance_w[0]);
        for (int j = 1; j < 7; ++j) clean = log_add(clean, t[j] + log(c_balance_w[j]));
        if (prior > 0.0) {
          double art = t[7] + log(c_theta_w[0] / H);
          for (int j = 1; j < 4 * H; ++j) art = log_add(art, t[7 + j] + log(c_theta_w[j / H] / H));
          out = log_add(log1p(-prior) + clean, log(prior) + art);
        } else {
          out = clean;
        }
      }
      gl[gl_off[g] + p] = out;
    }
    __syncthreads();
  }
}

// One thread per region: flags the regions whose best two genotypes lie within
// 1e-4 x max(1, reads) of each other, by GL or by GL plus the uniform
// haplotype prior (1 for a == b, 2 otherwise, normalised), as the numerical
// guard of caller/native/caller/partial_anchor.py:120-133 measures it.
__global__ void tie_kernel(const double* __restrict__ gl, const int64_t* __restrict__ gl_off,
                           const int32_t* __restrict__ region_h, const int64_t* __restrict__ region_reads,
                           int64_t n_regions, int* __restrict__ flags) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n_regions;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int H = region_h[g];
    const int P = H * (H + 1) / 2;
    if (P < 2) { flags[g] = 0; continue; }
    const double* v = gl + gl_off[g];
    const double lnH2 = 2.0 * log((double)H);
    double a1 = -HUGE_VAL, a2 = -HUGE_VAL, b1 = -HUGE_VAL, b2 = -HUGE_VAL;
    int p = 0;
    for (int b = 0; b < H; ++b)
      for (int a = 0; a <= b; ++a, ++p) {
        const double x = v[p];
        const double y = x + (a == b ? 0.0 : 0.6931471805599453094) - lnH2;
        if (x > a1) { a2 = a1; a1 = x; } else if (x > a2) { a2 = x; }
        if (y > b1) { b2 = b1; b1 = y; } else if (y > b2) { b2 = y; }
      }
    const double margin = 1e-4 * fmax(1.0, (double)region_reads[g]);
    flags[g] = fmin(a1 - a2, b1 - b2) <= margin ? 1 : 0;
  }
}

}  // namespace

cudaError_t launch_genotype_ties(const double* gl, const int64_t* gl_off, const int32_t* region_h,
                                 const int64_t* region_reads, int64_t n_regions, int* flags, cudaStream_t stream) {
  if (n_regions <= 0) return cudaSuccess;
  const int grid = (int)((n_regions + 255) / 256 < 1024 ? (n_regions + 255) / 256 : 1024);
  tie_kernel<<<grid, 256, 0, stream>>>(gl, gl_off, region_h, region_reads, n_regions, flags);
  return cudaGetLastError();
}

cudaError_t launch_genotype_rows(const double* ln, const int64_t* row_off, const int32_t* row_h,
                                 const double* mq_error, int64_t n_reads, double* values, double* certainty,
                                 int sm_count, cudaStream_t stream) {
  if (n_reads <= 0) return cudaSuccess;
  const int64_t blocks = (n_reads + 7) / 8;
  const int grid = (int)(blocks < (int64_t)sm_count * 16 ? blocks : (int64_t)sm_count * 16);
  rows_kernel<<<grid, 256, 0, stream>>>(ln, row_off, row_h, mq_error, n_reads, values, certainty);
  return cudaGetLastError();
}

cudaError_t launch_genotype_gl(const double* values, const int64_t* region_out_off, const int64_t* region_reads,
                               const int32_t* region_h, const int64_t* gl_off, const int64_t* acc_off,
                               int64_t n_regions, double prior, double* acc, double* gl, int sm_count,
                               cudaStream_t stream) {
  if (n_regions <= 0) return cudaSuccess;
  const int grid = (int)(n_regions < (int64_t)sm_count * 8 ? n_regions : (int64_t)sm_count * 8);
  gl_kernel<<<grid, 128, 0, stream>>>(values, region_out_off, region_reads, region_h, gl_off, acc_off, n_regions,
                                      prior, acc, gl);
  return cudaGetLastError();
}

}  // namespace vd
