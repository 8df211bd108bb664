// PairHMM forward pass on sm_100a: anti-diagonal wavefront, one warp per read.
//
// Model (VarDepth caller/native/caller/wide.cpp:9-33 semiglobal,
// anchored.cpp:5-25 anchored; g = gap-open, x = gap-continuation):
//   M[i][j] = E_ij ((1-2g) M[i-1][j-1] + (1-x)(I[i-1][j-1] + D[i-1][j-1]))
//   I[i][j] = (g M[i-1][j] + x I[i-1][j]) / 4
//   D[i][j] = g M[i][j-1] + x D[i][j-1]
//   E_ij = read[i-1]==hap[j-1] ? 1-e_i : e_i/3,  e = 10^(-min(q,60)/10)
//
// Work decomposition.  A warp owns one read (n rows) and streams through a list
// of K haplotypes.  Lane L owns R consecutive rows of the current strip of
// 32*R rows (reads longer than 256 bases are strip-mined with R = 8); the
// placement of the read in the strip is described at process_item.  At step
// t lane L is at position p = t - L of the "column stream": haplotype k
// occupies positions S_k (its column 0) .. S_k + m_k.  Consecutive haplotypes
// follow each other without a gap, so the 31-step wavefront ramp is paid once
// per read, not once per pair.  Lane L-1 hands its bottom row to lane L through
// two warp shuffles per step.
//
// Scaled variables.  Row i is multiplied by f_i = 1 / (a max(P1_i, P0_i))
// (a = 1-2g, P1 = 1-e, P0 = e/3) and by a power-of-two constant c, so that a
// matching cell costs no emission multiply.  With C_i = C_0 prod f_k:
//   mu_i = C_i M_i,   nu_i = C_i I_i / (alpha f_i)  (alpha = g/4),   om_i = C_i D_i / g
//   mu_i(j) = s_{i-1}(j-1) * (match ? hit_i : miss_i)        hit_i = 1 unless P0 > P1
//   nu_i(j) = u_{i-1}(j)
//   om_i(j) = mu_i(j-1) + x om_i(j-1)
//   u_i(j)  = mu_i(j) + X_i nu_i(j)                  X_i = (x/4) f_i
//   s_i(j)  = mu_i(j) + K_i nu_i(j) + k2 om_i(j)     K_i = k1 f_i, k1 = (1-x) alpha / a, k2 = (1-x) g / a
// which is 6 issue slots per cell (compare, predicated multiply, 4 FMA).
// The row factors are undone exactly in FP64 at the end:
//   ln Z = ln Zs - ln C_0 + sum_i ln N_i - E ln 2,   N_i = 1/f_i,
// E being the sum of the power-of-two strip renormalisations.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vd {

constexpr int kWarp = 32;
constexpr int kMaxR = 8;                       // read rows per lane
constexpr int kLongGroupMax = 8;               // haplotypes of one long-read warp item
constexpr int kStripRows = kWarp * kMaxR;      // rows per strip of a long read
constexpr int kWarpsPerBlock = 4;
constexpr int kDriftTier = 3;  // tier number of the FP32 drift-compensated rescue (pairhmm_kernel.cuh)

// Work item: one read against a list of haplotypes.
struct WorkItem {
  int32_t read;       // read index
  int32_t nhap;       // haplotypes in the list
  int64_t hap_begin;  // first haplotype (contiguous lists) or offset into hap_sel
  int64_t out_begin;  // output slot of the first haplotype, or offset into out_sel
  int32_t code;       // R | general << 8 | multistrip << 9 | paired << 10 | long << 11
  int32_t read2;      // second read of a paired item (same region and R), else -1
  int64_t out2_begin; // output slot of the second read's first haplotype
};

// A pair sent to the next precision tier.
struct RescueEntry {
  int32_t read;
  int32_t hap;
  int64_t out;
};

inline __host__ __device__ int code_R(int c) { return c & 15; }
inline __host__ __device__ bool code_general(int c) { return (c >> 8) & 1; }
inline __host__ __device__ bool code_paired(int c) { return (c >> 10) & 1; }
inline __host__ __device__ int make_code(int R, bool general, bool multistrip) {
  return R | (general ? 256 : 0) | (multistrip ? 512 : 0);
}
constexpr int kPairedBit = 1024;
constexpr int kLongBit = 2048;  // a long read against one or two haplotypes (pairhmm_long.cuh)
inline __host__ __device__ bool code_long(int c) { return (c >> 11) & 1; }

// Per-quality tables (index = raw Phred byte) and scalar constants for one
// (gap, ext, offsets) setting, in the arithmetic type of the kernel.
template <typename T>
struct Tables {
  T hit[256];    // match factor  P1 / max(P1, P0)
  T miss[256];   // mismatch factor P0 / max(P1, P0)
  T K[256];      // k1 * f
  T X[256];      // (x/4) * f
  T A[256];      // alpha * f   (weight of nu in the final row sums)
  double lnN[256];  // ln(a max(P1, P0))
  unsigned char general[256];  // P0 > P1: needs the two-sided emission select
};

template <typename T>
struct Scalars {
  T k2, x, gfin, c;          // c: value of the row-0 cells (power of two)
  double ln_c;               // ln c
  T strip_floor;             // below this a strip boundary counts as underflowed
  T strip_ceil;              // at or above this it counts as overflowed (+inf: only inf / NaN)
  T final_floor;             // below this the final scaled sum counts as underflowed
  int target_log2;           // strip boundary maxima are renormalised to 2^target
};

// Device-side view of one batch.
struct BatchView {
  const uint8_t* read_bases;
  const uint8_t* read_quals;
  const int64_t* read_off;    // [n_reads + 1]
  const int32_t* read_code;   // per read: make_code(...) of its primary tier
  const uint8_t* hap_bases;
  const int64_t* hap_off;     // [n_haps + 1]
  const int32_t* hap_sel;     // nullable: indirect haplotype lists
  const int64_t* out_sel;     // nullable: indirect output slots
  double* out;
  const int32_t* hap_order;   // nullable: two-read items read their haplotypes through it (a
                              // region's haplotypes in lexicographic order; the entry is the
                              // chunk-local haplotype and, added to out_begin, the output slot)
  const int32_t* hap_share;   // nullable, same positions: Q >= 0 when the haplotype shares DP
                              // columns 0..Q with the one before it
};

struct QueueView {
  const WorkItem* items;      // nullable when the list is a rescue list
  const RescueEntry* entries; // rescue input (tiers 1 and 2)
  const unsigned long long* count;  // number of entries (device, rescue tiers)
  long long n_items;          // number of items (primary tier)
  unsigned long long* head;   // work counter (reset to 0 before launch)
  RescueEntry* spill;         // output rescue list for the next tier
  unsigned long long* spill_count;
  long long spill_cap;
  void* scratch;              // strip boundaries: per warp slot, scratch_stride elements
  long long scratch_stride;   // in boundary records (float2 / double2)
  int* error_flag;            // set when the spill list overflows
  int static_order;           // 1: warp w takes items w, w + W, w + 2W ... (W = warps in the grid)
  unsigned long long* strip_runs;  // long-read kernel, nullable: [0] runs of strips, [1] strips
};

}  // namespace vd
