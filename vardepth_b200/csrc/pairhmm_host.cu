// Host side of the B200 PairHMM: engine, work-list construction, memory-budget
// batching, tier orchestration (FP32 -> FP64 -> FP64 32-row strips), CUDA
// graph replay of resident plans, and the C ABI declared in
// include/vardepth_pairhmm.h.
//
// Dispatch semantics follow caller/native/caller/accelerator.py:105-159
// (CudaPairHMM.score): validate, bucket, chunk by a device-memory budget,
// transfer, launch, copy back, and re-score the pairs the reduced-precision
// pass could not resolve.  Here the re-scoring runs on the GPU as two further
// kernel tiers fed by device-side lists, so a batch needs no host round trip.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/vardepth_pairhmm.h"
#include "pairhmm_core.cuh"
#include "pairhmm_launch.h"
#include "pairhmm_backward.cuh"

using namespace vd;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  // consume the thread's last-error slot so a later launch check does not
  // report this (non-sticky) error again
  cudaGetLastError();
  return fail(VD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define VD_CUDA(call)                                   \
  do {                                                  \
    cudaError_t vd_err_ = (call);                       \
    if (vd_err_ != cudaSuccess) return cuda_fail(vd_err_, #call); \
  } while (0)

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Runs fn(begin, end) over [0, n) in contiguous slices on up to 32 host threads
// (the calling thread takes the first slice); ranges below 2 grains run inline.
template <typename F>
void parallel_for(int64_t n, int64_t grain, F&& fn) {
  const int64_t hw = std::max<int64_t>(1, (int64_t)std::thread::hardware_concurrency());
  const int64_t T = std::min<int64_t>(std::min<int64_t>(hw, 32), std::max<int64_t>(1, n / std::max<int64_t>(1, grain)));
  if (T <= 1) { fn((int64_t)0, n); return; }
  std::vector<std::thread> th;
  th.reserve((size_t)T - 1);
  for (int64_t t = 1; t < T; ++t) th.emplace_back([&fn, n, t, T] { fn(n * t / T, n * (t + 1) / T); });
  fn((int64_t)0, n / T);
  for (auto& x : th) x.join();
}

// ---- model tables -----------------------------------------------------------

int quality_bin(unsigned q) {
  if (q < 15u) return 0;
  if (q < 25u) return 1;
  if (q < 35u) return 2;
  return 3;
}

struct TableSet {
  Tables<float> f32;
  Tables<double> f64;
  Scalars<float> s32;
  Scalars<double> s64;
  Scalars<float> s32d;  // the drift tier: row 0 = 1, strips brought to 2^0, window 2^-60 .. 2^60
};

// Per-quality factors of the scaled recurrence (pairhmm_core.cuh).  The error
// of a Phred byte is 10^(-min(q,60)/10) (accelerator.py:23), optionally
// shifted by the bin offset.
void build_tables(double g, double x, const double* offsets, TableSet* ts) {
  const double a = 1.0 - 2.0 * g, b = 1.0 - x, alpha = 0.25 * g;
  const double k1 = b * alpha / a, k2 = b * g / a, x4 = 0.25 * x;
  for (int q = 0; q < 256; ++q) {
    double phred = (double)std::min(q, 60);
    if (offsets) phred = std::max(0.0, phred + offsets[quality_bin((unsigned)q)]);
    const double e = std::pow(10.0, -phred / 10.0);
    const double p1 = 1.0 - e, p0 = e / 3.0;
    const double mx = std::max(p1, p0);
    const double N = a * mx, f = 1.0 / N;
    const double hit = p1 / mx, miss = p0 / mx, K = k1 * f, X = x4 * f, A = alpha * f;
    ts->f32.hit[q] = (float)hit;  ts->f64.hit[q] = hit;
    ts->f32.miss[q] = (float)miss; ts->f64.miss[q] = miss;
    ts->f32.K[q] = (float)K;      ts->f64.K[q] = K;
    ts->f32.X[q] = (float)X;      ts->f64.X[q] = X;
    ts->f32.A[q] = (float)A;      ts->f64.A[q] = A;
    ts->f32.lnN[q] = std::log(N); ts->f64.lnN[q] = std::log(N);
    const unsigned char gen = p0 > p1 ? 1 : 0;
    ts->f32.general[q] = gen;     ts->f64.general[q] = gen;
  }
  ts->s32.k2 = (float)k2; ts->s32.x = (float)x; ts->s32.gfin = (float)g;
  // FP32 range: cells stay below ~1.33 c (a row grows by at most 1 + K + k2/(1-x)
  // ~ 1.0011 over its predecessor), so c = 2^120 leaves 2^7 of headroom; a final
  // sum >= 2^-80 keeps the dominant cells normal (>= 2^-93 after m+1 <= 2^13 terms)
  ts->s32.c = std::ldexp(1.0f, 120); ts->s32.ln_c = 120.0 * std::log(2.0);
  ts->s32.strip_floor = std::ldexp(1.0f, -40); ts->s32.final_floor = std::ldexp(1.0f, -80);
  ts->s32.strip_ceil = HUGE_VALF;
  ts->s32.target_log2 = 120;
  // the drift tier keeps every strip's bottom near 2^0 with per-row boosts, so
  // it starts there and leaves 60 binary orders either side for what the
  // boosts do not cancel
  ts->s32d = ts->s32;
  ts->s32d.c = 1.0f; ts->s32d.ln_c = 0.0;
  ts->s32d.strip_floor = std::ldexp(1.0f, -60); ts->s32d.strip_ceil = std::ldexp(1.0f, 60);
  ts->s32d.final_floor = std::ldexp(1.0f, -60);
  ts->s32d.target_log2 = 0;
  ts->s64.k2 = k2; ts->s64.x = x; ts->s64.gfin = g;
  ts->s64.c = std::ldexp(1.0, 600); ts->s64.ln_c = 600.0 * std::log(2.0);
  ts->s64.strip_floor = std::ldexp(1.0, -800); ts->s64.final_floor = std::ldexp(1.0, -900);
  ts->s64.strip_ceil = HUGE_VAL;
  ts->s64.target_log2 = 600;
}

struct TableKey {
  double g, x, off[4];
  bool has_off;
  bool operator==(const TableKey& o) const {
    if (g != o.g || x != o.x || has_off != o.has_off) return false;
    if (has_off) for (int i = 0; i < 4; ++i) if (off[i] != o.off[i]) return false;
    return true;
  }
};

// ---- device buffers -----------------------------------------------------------

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  int reserve(size_t n) {
    if (n <= bytes) return VD_OK;
    if (p) { cudaFree(p); p = nullptr; bytes = 0; }
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) { cudaGetLastError(); return fail(VD_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e)); }
    bytes = n;
    return VD_OK;
  }
};

}  // namespace

// ---- engine -----------------------------------------------------------------------

struct vd_engine {
  int device = 0;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  char name[256] = {0};
  size_t budget = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_mid = nullptr, ev_end = nullptr;
  // the long-read kernel runs on a side stream beside the other primary
  // kernels: as its persistent blocks run out of items, theirs take the SMs
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::mutex mu;
  int grid[2][2] = {{0, 0}, {0, 0}};  // [f64][anchored] blocks
  int grid_pair[2][2] = {{0, 0}, {0, 0}};  // blocks of the two-read kernels [split == 7][wide]
  int grid_drift = 0;                 // blocks of the drift tier (no more than grid[0][0])
  int grid_long[2][2] = {{0, 0}, {0, 0}};  // blocks of the long-read kernels [block][R == 8] (<= grid[0][0])
  int grid_grad[2] = {0, 0};          // blocks of the gradient kernel [f64]
  vd_tuning tuning{256, 0x1fe, 0, 0, VD_LONG_WARP, 6, kLongGroupMax, {0}};  // vd_engine_set_tuning
  DevBuf grad_arena;                  // inputs, lists and scratch of vd_forward_backward
  DevBuf geno_arena;                  // buffers of vd_region_genotypes
  // table cache
  TableKey tkey{};
  bool tvalid = false;
  TableSet* htab = nullptr;   // pinned host copy
  DevBuf dtab;
  // batch arena reused by vd_forward
  DevBuf arena;
  std::vector<double> out_stage;
  // live plans: destroying the engine first releases their device resources
  std::unordered_set<vd_plan*> plans;
  // vd_forward pipeline: two slots, each with its own stream, arena and events,
  // so one chunk's host work-list build and upload overlap the other's kernels
  struct Slot {
    DevBuf arena;
    cudaStream_t stream = nullptr, side = nullptr;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork = nullptr, join = nullptr;
    unsigned long long* hcnt = nullptr;  // pinned copy of the tier counters
    std::vector<double> stage;           // pair-form outputs before the scatter
    vd_plan* pl = nullptr;
    bool busy = false;
    int launches = 0;
  };
  Slot slots[2];
};

namespace {

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) { if (cudaGetDevice(&prev) != cudaSuccess) prev = -1; cudaSetDevice(dev); }
  ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

int ensure_tables(vd_engine* e, const vd_params* p) {
  TableKey k{};
  k.g = p->gap; k.x = p->ext; k.has_off = p->quality_offsets != nullptr;
  if (k.has_off) for (int i = 0; i < 4; ++i) k.off[i] = p->quality_offsets[i];
  if (e->tvalid && k == e->tkey) return VD_OK;
  build_tables(p->gap, p->ext, p->quality_offsets, e->htab);
  int rc = e->dtab.reserve(sizeof(TableSet));
  if (rc) return rc;
  VD_CUDA(cudaMemcpyAsync(e->dtab.p, e->htab, sizeof(TableSet), cudaMemcpyHostToDevice, e->stream));
  VD_CUDA(cudaStreamSynchronize(e->stream));
  e->tkey = k;
  e->tvalid = true;
  return VD_OK;
}

int validate_params(const vd_params* p) {
  if (!p) return fail(VD_EINVAL, "params is NULL");
  if (!(p->gap >= 0.0 && p->gap < 0.5)) return fail(VD_EINVAL, "gap must lie in [0, 0.5)");
  if (!(p->ext >= 0.0 && p->ext < 1.0)) return fail(VD_EINVAL, "ext must lie in [0, 1)");
  if (p->anchored != 0 && p->anchored != 1) return fail(VD_EINVAL, "anchored must be 0 or 1");
  if (p->precision != VD_PRECISION_MIXED && p->precision != VD_PRECISION_FLOAT64)
    return fail(VD_EINVAL, "unknown precision");
  if (p->quality_offsets)
    for (int i = 0; i < 4; ++i)
      if (!std::isfinite(p->quality_offsets[i])) return fail(VD_EINVAL, "quality offsets must be finite");
  if (p->schedule != VD_SCHEDULE_BATCHED && p->schedule != VD_SCHEDULE_PLAIN)
    return fail(VD_EINVAL, "unknown schedule");
  for (int i = 0; i < 3; ++i) if (p->reserved[i]) return fail(VD_EINVAL, "reserved fields must be zero");
  return VD_OK;
}

bool offsets_ok(const int64_t* off, int64_t n) {
  if (n < 0 || !off) return false;
  if (off[0] < 0) return false;
  for (int64_t i = 0; i < n; ++i) if (off[i + 1] < off[i] || off[i + 1] - off[i] > (1 << 28)) return false;
  return true;
}

int validate_batch(const vd_batch* b) {
  if (!b) return fail(VD_EINVAL, "batch is NULL");
  if (b->n_reads < 0 || b->n_haps < 0) return fail(VD_EINVAL, "negative counts");
  if (b->n_reads > INT32_MAX - 1 || b->n_haps > INT32_MAX - 1) return fail(VD_EINVAL, "too many reads or haplotypes");
  if (!offsets_ok(b->read_off, b->n_reads)) return fail(VD_EINVAL, "read offsets must be non-decreasing (lengths <= 2^28)");
  if (!offsets_ok(b->hap_off, b->n_haps)) return fail(VD_EINVAL, "haplotype offsets must be non-decreasing (lengths <= 2^28)");
  if (b->read_off[b->n_reads] > b->read_off[0] && (!b->read_bases || !b->read_quals))
    return fail(VD_EINVAL, "read buffers are NULL");
  if (b->hap_off[b->n_haps] > b->hap_off[0] && !b->hap_bases) return fail(VD_EINVAL, "haplotype buffer is NULL");
  if (b->pair_read) {
    if (!b->pair_hap || b->n_pairs < 0) return fail(VD_EINVAL, "pair arrays inconsistent");
    for (int64_t p = 0; p < b->n_pairs; ++p)
      if (b->pair_read[p] < 0 || b->pair_read[p] >= b->n_reads || b->pair_hap[p] < 0 || b->pair_hap[p] >= b->n_haps)
        return fail(VD_EINVAL, "pair index out of range");
  } else {
    if (b->n_regions < 0 || !b->region_read_off || !b->region_hap_off) return fail(VD_EINVAL, "region arrays missing");
    for (int64_t g = 0; g < b->n_regions; ++g) {
      if (b->region_read_off[g + 1] < b->region_read_off[g] || b->region_hap_off[g + 1] < b->region_hap_off[g])
        return fail(VD_EINVAL, "region offsets must be non-decreasing");
    }
    if (b->n_regions > 0) {
      if (b->region_read_off[0] < 0 || b->region_read_off[b->n_regions] > b->n_reads ||
          b->region_hap_off[0] < 0 || b->region_hap_off[b->n_regions] > b->n_haps)
        return fail(VD_EINVAL, "region offsets out of range");
    }
  }
  return VD_OK;
}

int64_t batch_outputs(const vd_batch* b) {
  if (b->pair_read) return b->n_pairs;
  int64_t total = 0;
  for (int64_t g = 0; g < b->n_regions; ++g)
    total += (b->region_read_off[g + 1] - b->region_read_off[g]) * (b->region_hap_off[g + 1] - b->region_hap_off[g]);
  return total;
}

// Work-list choices the engine's tuning sets (vd_tuning).
struct BuildOpts {
  int long_R = kMaxR;              // rows per lane of reads longer than one 256-row strip
  bool long_warp = true;           // such reads (FP32 semiglobal) run a read against two haplotypes per item
  bool long_block = false;         // ... on a block per item (the CTA's warps split each strip)
  int long_group = kLongGroupMax;  // haplotypes per warp item of such a read
  int pair_split = 6;              // two-read items with this many rows per lane or more: 12-warp kernel
  int pair_mask = 0x1fe;           // bit R: two reads of R rows per lane may share a warp
  int64_t max_stream = 1 << 30;    // haplotype columns one work item streams at most
};

// Rows per lane for a read of n rows: the smallest R with 32 R >= n, at most
// 8; longer reads are strip-mined in strips of 32 long_R rows.
int rows_per_lane(int n, int long_R = kMaxR) {
  if (n > kStripRows) return long_R;
  return std::min(kMaxR, std::max(1, (n + kWarp - 1) / kWarp));
}

BuildOpts build_opts(const vd_engine* e) {
  BuildOpts bo;
  bo.long_R = e->tuning.long_read_rows / kWarp;
  bo.pair_mask = e->tuning.pair_mask;
  bo.max_stream = e->tuning.max_item_columns > 0 ? (int64_t)e->tuning.max_item_columns : (int64_t)1 << 30;
  bo.long_warp = (e->tuning.long_mode == VD_LONG_WARP || e->tuning.long_mode == VD_LONG_BLOCK) &&
                 (bo.long_R == 8 || bo.long_R == 4);
  bo.long_block = e->tuning.long_mode == VD_LONG_BLOCK;
  bo.long_group = bo.long_block ? 2 : e->tuning.long_group > 0 ? e->tuning.long_group : kLongGroupMax;
  bo.pair_split = e->tuning.pair_split == 7 ? 7 : 6;
  return bo;
}


// ---- host plan ------------------------------------------------------------------

// A chunk of a batch laid out the way the kernels read it.
struct HostChunk {
  // reads [ra, rb) and haplotypes [ha, hb) of the batch (global indices)
  int64_t ra = 0, rb = 0, ha = 0, hb = 0;
  std::vector<int64_t> read_off;   // rebased, rb - ra + 1
  std::vector<int32_t> read_code;
  std::vector<int64_t> hap_off;    // rebased, hb - ha + 1
  std::vector<WorkItem> items;
  std::vector<int32_t> hap_sel;    // pair form
  std::vector<int64_t> out_sel;    // pair form (chunk-local output slots)
  std::vector<int64_t> out_global; // pair form: batch output index of each local slot
  std::vector<int32_t> hap_order;  // region form, two-read items: chunk-local haplotype at each position
                                   // (every region's haplotypes in lexicographic order)
  std::vector<int32_t> hap_share;  // the same positions: shared prefix column with the previous one
  int64_t out_begin = 0;           // region form: first batch output slot
  int64_t n_out = 0;
  int64_t cells = 0;
  int64_t shared_cells = 0;        // of cells, those two-read items skip by prefix sharing
  int64_t pairs_scored = 0;
  int max_hap = 0;
  bool any_long = false;           // a read longer than 32 (the robust tier strip-mines it)
  bool any_strip = false;          // a read longer than one 256-row strip (every tier strip-mines it)
  int64_t n_paired = 0;            // leading items that carry two reads (own kernels)
  int64_t n_paired_wide = 0;       // the first of them, with pair_split..8 rows per lane
  int pair_split = 6;              // rows per lane from which two-read items run at 12 warps per SM
  int64_t n_long = 0;              // the items after them: long reads, two haplotypes per item
  int long_R = kMaxR;              // rows per lane of those
  bool long_block = false;         // and their kernel: block per item (else warp per item)
};

// The robust tier runs on a small grid: it only sees pairs the FP64 wavefront
// could not resolve, and its strip scratch then stays small.
constexpr int kRobustBlocks = 32;

// Order the work list for the persistent warps.  Items are grouped by kernel
// variant (the code: rows per lane, final-row register, emission form) so that
// the warps resident on an SM run the same unrolled loop at the same time --
// interleaving variants thrashes the instruction cache -- and inside a group
// they run longest-processing-time first.  Groups with the largest items come
// first, so the tail of the whole list holds the smallest items.  O(n) passes.
void order_items(std::vector<WorkItem>& items, const std::vector<int64_t>& cost) {
  const size_t n = items.size();
  if (n < 2) return;
  // cost bucket (descending) inside a group
  const int nb = 256;
  std::vector<int> bucket(n);
  for (size_t i = 0; i < n; ++i) {
    // quarter-octave bucket: floor(log2 c) and the next two bits
    const uint64_t c = (uint64_t)std::max<int64_t>(4, cost[i]);
    const int lz = 63 - __builtin_clzll(c);
    int k = lz * 4 + (int)((c >> (lz - 2)) & 3);
    k = std::max(0, std::min(nb - 1, k));
    bucket[i] = nb - 1 - k;
  }
  // groups ordered by decreasing mean cost (codes are small integers)
  constexpr int kCodes = 4096;
  std::vector<double> sum(kCodes, 0.0);
  std::vector<int64_t> cnt(kCodes, 0);
  for (size_t i = 0; i < n; ++i) {
    const int cd = items[i].code & (kCodes - 1);
    sum[cd] += (double)cost[i];
    cnt[cd] += 1;
  }
  std::vector<std::pair<double, int32_t>> groups;
  for (int cd = 0; cd < kCodes; ++cd)
    if (cnt[cd]) groups.push_back({sum[cd] / (double)cnt[cd], cd});
  std::sort(groups.begin(), groups.end(), [](auto& a, auto& b) { return a.first > b.first || (a.first == b.first && a.second < b.second); });
  std::vector<int> rank(kCodes, 0);
  for (size_t g = 0; g < groups.size(); ++g) rank[groups[g].second] = (int)g;
  const int ng = (int)groups.size();
  std::vector<int64_t> count((size_t)ng * nb + 1, 0);
  std::vector<int64_t> key(n);
  for (size_t i = 0; i < n; ++i) {
    key[i] = (int64_t)rank[items[i].code & (kCodes - 1)] * nb + bucket[i];
    ++count[key[i] + 1];
  }
  for (size_t k = 0; k + 1 < count.size(); ++k) count[k + 1] += count[k];
  std::vector<WorkItem> out(n);
  for (size_t i = 0; i < n; ++i) out[count[key[i]]++] = items[i];
  items.swap(out);
}

struct ReadInfo {
  int n;
  int32_t code;
};

ReadInfo read_info(const vd_batch* b, int64_t r, bool anchored, int long_R = kMaxR) {
  const int64_t o = b->read_off[r];
  const int n = (int)(b->read_off[r + 1] - o);
  ReadInfo ri{n, 0};
  if (n <= 0) return ri;
  // P0 > P1 only for Phred 0 and 1 (e > 0.75); offsets can move a bin there.
  // A branch-free minimum vectorises; an early exit would not.
  const unsigned char* q = b->read_quals + o;
  unsigned char qmin = 255;
  for (int i = 0; i < n; ++i) qmin = q[i] < qmin ? q[i] : qmin;
  const bool gen = qmin < 2;
  // anchored reads carry one extra row on top: the emulator of row 0
  const int rows = n + (anchored ? 1 : 0);
  ri.code = make_code(rows_per_lane(rows, long_R), gen, rows > kStripRows);
  return ri;
}

// Quality offsets can push bins into the P0 > P1 regime; recompute the
// general flag from the tables in that case.
bool read_general(const vd_batch* b, int64_t r, const TableSet* ts) {
  const int64_t o = b->read_off[r];
  const int n = (int)(b->read_off[r + 1] - o);
  for (int i = 0; i < n; ++i) if (ts->f64.general[b->read_quals[o + i]]) return true;
  return false;
}

void finish_chunk_common(HostChunk& c, const vd_batch* b, const TableSet* ts, bool offsets, bool anchored,
                         const BuildOpts& bo = BuildOpts()) {
  c.read_off.resize(c.rb - c.ra + 1);
  c.read_code.resize(c.rb - c.ra);
  const int64_t r0 = b->read_off[c.ra];
  parallel_for(c.rb - c.ra, 4096, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) {
      const int64_t r = c.ra + k;
      c.read_off[k] = b->read_off[r] - r0;
      ReadInfo ri = read_info(b, r, anchored, bo.long_R);
      if (offsets && ri.n > 0 && !code_general(ri.code) && read_general(b, r, ts))
        ri.code |= 256;
      c.read_code[k] = ri.code;
    }
  });
  c.read_off[c.rb - c.ra] = b->read_off[c.rb] - r0;
  for (int64_t r = c.ra; r < c.rb; ++r) {
    const int n = (int)(b->read_off[r + 1] - b->read_off[r]);
    const int rows = n + (anchored ? 1 : 0);
    if (n > 0 && rows > kWarp) c.any_long = true;
    if (n > 0 && rows > kStripRows) c.any_strip = true;
  }
  c.hap_off.resize(c.hb - c.ha + 1);
  const int64_t h0 = b->hap_off[c.ha];
  for (int64_t h = c.ha; h <= c.hb; ++h) c.hap_off[h - c.ha] = b->hap_off[h] - h0;
  c.max_hap = 0;
  for (int64_t h = c.ha; h < c.hb; ++h) c.max_hap = std::max<int>(c.max_hap, (int)(b->hap_off[h + 1] - b->hap_off[h]));
}

// Shared haplotype prefixes of one region (two-read items).  The two-read
// items visit a region's haplotypes in lexicographic order (order[i], i over
// the region's positions), the depth-first order of their prefix tree, so each
// haplotype follows the one it shares most with.  share[i] = Q >= 0 says that
// the haplotype at position i agrees with the one at i-1 on its first Q
// bases, so DP columns 0..Q of the two are the same and the two-read kernel
// starts it at column Q+1 from the lane states it laid down at column Q of
// the previous one.  Each warp holds one such snapshot, so Q is used when the
// snapshot can be taken while the previous haplotype streams (Q at or past
// the column that one itself started from) or when it is still there (Q
// equal to the previous share); otherwise -1.  Q stays below the length of
// the haplotype (it streams at least one column) and at or above
// kMinShareColumns: a snapshot puts 32 steps of the ramp loop into the
// haplotype that takes it.
constexpr int kMinShareColumns = 32;

void region_order_and_shares(const vd_batch* b, int64_t h_lo, int64_t h_hi, int64_t ha, int32_t* order,
                             int32_t* share) {
  const int64_t nh = h_hi - h_lo;
  for (int64_t i = 0; i < nh; ++i) order[i] = (int32_t)(h_lo - ha + i);
  auto bytes = [&](int32_t lh) {
    const int64_t h = ha + lh;
    return std::make_pair(b->hap_bases + b->hap_off[h], (size_t)(b->hap_off[h + 1] - b->hap_off[h]));
  };
  std::stable_sort(order, order + nh, [&](int32_t x, int32_t y) {
    const auto [px, nx] = bytes(x);
    const auto [py, ny] = bytes(y);
    const int c = nx && ny ? std::memcmp(px, py, std::min(nx, ny)) : 0;
    return c != 0 ? c < 0 : nx < ny;
  });
  int prev_q = -1;
  for (int64_t i = 0; i < nh; ++i) {
    int q = -1;
    if (i > 0) {
      const auto [pa, ma] = bytes(order[i - 1]);
      const auto [pb, mb] = bytes(order[i]);
      if (ma > 0 && mb > 0) {
        const int lim = (int)std::min(ma, mb - 1);
        int l = 0;
        while (l < lim && pa[l] == pb[l]) ++l;
        if (l >= prev_q + 1) q = l;
        else if (prev_q >= 0 && l >= prev_q) q = prev_q;
        if (q < kMinShareColumns) q = -1;
      }
    }
    share[i] = q;
    prev_q = q;
  }
}

// Work items of a region chunk: one item per read with the region's non-empty
// haplotypes as contiguous runs; reads longer than a strip get one item per
// haplotype (their strip boundary scratch holds one haplotype).  With
// pair_reads, two reads of a region with the same kernel variant (single strip,
// one-sided emission) share an item and run in the packed two-read path.
// With plain (the comparison schedule) every pair is its own item with the
// fixed tile of kMaxR rows per lane, the list stays in input order and no
// reads are paired.
void build_region_chunk(const vd_batch* b, int64_t g0, int64_t g1, const TableSet* ts, bool offsets,
                        bool anchored, bool pair_reads, HostChunk& c, bool plain = false,
                        const BuildOpts& bo = BuildOpts()) {
  const bool fp32 = pair_reads;  // mixed precision: the FP32 kernels run the primary tier
  if (plain) pair_reads = false;
  c.long_R = bo.long_R;
  c.long_block = bo.long_block;
  c.ra = b->region_read_off[g0];
  c.rb = b->region_read_off[g1];
  c.ha = b->region_hap_off[g0];
  c.hb = b->region_hap_off[g1];
  c.out_begin = 0;
  for (int64_t g = 0; g < g0; ++g)
    c.out_begin += (b->region_read_off[g + 1] - b->region_read_off[g]) * (b->region_hap_off[g + 1] - b->region_hap_off[g]);
  finish_chunk_common(c, b, ts, offsets, anchored, bo);
  const int64_t kMaxStream = bo.max_stream;
  // output offset of every region inside the chunk
  const int64_t ng = g1 - g0;
  std::vector<int64_t> region_out_of(ng + 1, 0);
  for (int64_t k = 0; k < ng; ++k)
    region_out_of[k + 1] = region_out_of[k] + (b->region_read_off[g0 + k + 1] - b->region_read_off[g0 + k]) *
                                                  (b->region_hap_off[g0 + k + 1] - b->region_hap_off[g0 + k]);
  // regions are cut into a fixed number of slices (so the result does not
  // depend on the thread count) and the slices are built in parallel
  struct Slice {
    std::vector<WorkItem> items;
    std::vector<int64_t> cost;
    int64_t cells = 0, shared = 0, pairs = 0;
  };
  const int64_t nslices = std::max<int64_t>(1, std::min<int64_t>(256, ng / 16));
  std::vector<Slice> slices((size_t)nslices);
  const bool sharing = pair_reads && !anchored && !plain;
  c.hap_share.clear();
  c.hap_order.clear();
  if (sharing) {
    c.hap_share.assign((size_t)(c.hb - c.ha), -1);
    c.hap_order.assign((size_t)(c.hb - c.ha), 0);
  }
  parallel_for(nslices, 1, [&](int64_t s_lo, int64_t s_hi) {
   for (int64_t si = s_lo; si < s_hi; ++si) {
    Slice& sl = slices[(size_t)si];
    std::vector<WorkItem>& items = sl.items;
    std::vector<int64_t>& cost = sl.cost;
    for (int64_t g = g0 + ng * si / nslices; g < g0 + ng * (si + 1) / nslices; ++g) {
    const int64_t r_lo = b->region_read_off[g], r_hi = b->region_read_off[g + 1];
    const int64_t h_lo = b->region_hap_off[g], h_hi = b->region_hap_off[g + 1];
    const int64_t nh = h_hi - h_lo;
    const int64_t region_out = region_out_of[g - g0];
    if (sharing)
      region_order_and_shares(b, h_lo, h_hi, c.ha, c.hap_order.data() + (h_lo - c.ha),
                              c.hap_share.data() + (h_lo - c.ha));
    // a long read (FP32 semiglobal, one-sided emission) against its region's
    // non-empty haplotypes: runs of up to long_group neighbours per item, in
    // both schedules (the haplotypes after an item's first pair take their
    // boosts from it, so the grouping is part of the result)
    auto emit_long = [&](int64_t r) {
      const int32_t code = c.read_code[r - c.ra];
      const int n = (int)(c.read_off[r - c.ra + 1] - c.read_off[r - c.ra]);
      const int64_t rows = (int64_t)kWarp * bo.long_R * ((n + kWarp * bo.long_R - 1) / (kWarp * bo.long_R));
      auto len = [&](int64_t h) { return (int)(b->hap_off[h + 1] - b->hap_off[h]); };
      for (int64_t h = h_lo; h < h_hi;) {
        if (len(h) <= 0) { ++h; continue; }
        int k = 1;
        while (k < bo.long_group && h + k < h_hi && len(h + k) > 0) ++k;
        int64_t work = 0, cells = 0;
        for (int j = 0; j < k; j += 2) {
          const int ma = len(h + j), mb = j + 1 < k ? len(h + j + 1) : 0;
          work += rows * (std::max(ma, mb) + 1 + kWarp) * (j + 1 < k ? 2 : 1);
          cells += (int64_t)n * (ma + mb);
        }
        WorkItem w;
        w.read = (int32_t)(r - c.ra);
        w.nhap = k;
        w.hap_begin = h - c.ha;
        w.out_begin = region_out + (r - r_lo) * nh + (h - h_lo);
        w.code = (code & ~15) | bo.long_R | kLongBit;
        w.read2 = -1;
        w.out2_begin = 0;
        items.push_back(w);
        cost.push_back(work);
        sl.cells += cells;
        sl.pairs += k;
        h += k;
      }
    };
    // emit the haplotype runs of read r (and r2 >= 0 riding along)
    auto emit = [&](int64_t r, int64_t r2) {
      const int32_t code = c.read_code[r - c.ra];
      const int n = (int)(c.read_off[r - c.ra + 1] - c.read_off[r - c.ra]);
      const int n2 = r2 >= 0 ? (int)(c.read_off[r2 - c.ra + 1] - c.read_off[r2 - c.ra]) : 0;
      // the plain schedule's fixed tile is 8 rows per lane; reads longer than a
      // strip keep the tuned strip height in both schedules (same strips, same bits)
      const bool fixed_tile = plain && (code & 512) == 0;
      const int R = fixed_tile ? kMaxR : code_R(code);
      const int item_code = fixed_tile ? (code & ~15) | kMaxR : code;
      const int n_rows = n + (anchored ? 1 : 0);
      const int64_t rows = (int64_t)kWarp * R * ((n_rows + kWarp * R - 1) / (kWarp * R));
      const bool multistrip = n_rows > kStripRows;
      // two-read items walk the region in its lexicographic order: position
      // i (global numbering) holds haplotype hap_at(i)
      const bool sorted = r2 >= 0 && sharing;
      auto hap_at = [&](int64_t i) -> int64_t { return sorted ? c.ha + c.hap_order[i - c.ha] : i; };
      auto len_at = [&](int64_t i) -> int { const int64_t x = hap_at(i); return (int)(b->hap_off[x + 1] - b->hap_off[x]); };
      int64_t h = h_lo;
      while (h < h_hi) {
        const int m0 = len_at(h);
        if (m0 <= 0) { ++h; continue; }
        int64_t run_end = h, stream = 0;
        while (run_end < h_hi) {
          const int m = len_at(run_end);
          if (m <= 0) break;
          // a haplotype after the first of a two-read run streams only the
          // columns past its shared prefix
          const int col0 = (sorted && run_end > h) ? c.hap_share[run_end - c.ha] + 1 : 0;
          if (run_end > h && (plain || multistrip || stream + m + 1 - col0 > kMaxStream)) break;
          stream += m + 1 - col0;
          sl.cells += (int64_t)(n + n2) * m;
          if (col0 > 0) sl.shared += (int64_t)(n + n2) * (col0 - 1);
          sl.pairs += r2 >= 0 ? 2 : 1;
          ++run_end;
        }
        WorkItem w;
        w.read = (int32_t)(r - c.ra);
        w.nhap = (int32_t)(run_end - h);
        w.hap_begin = h - c.ha;
        // sorted: output slot = out_begin + hap_order[position] (the chunk-local haplotype)
        const int64_t col = sorted ? -(h_lo - c.ha) : (h - h_lo);
        w.out_begin = region_out + (r - r_lo) * nh + col;
        w.code = r2 >= 0 ? (item_code | kPairedBit) : item_code;
        w.read2 = r2 >= 0 ? (int32_t)(r2 - c.ra) : -1;
        w.out2_begin = r2 >= 0 ? region_out + (r2 - r_lo) * nh + col : 0;
        items.push_back(w);
        cost.push_back(rows * (stream + kWarp) * (r2 >= 0 ? 2 : 1));
        h = run_end;
      }
    };
    int64_t waiting[kMaxR + 1];
    for (int k = 0; k <= kMaxR; ++k) waiting[k] = -1;
    for (int64_t r = r_lo; r < r_hi; ++r) {
      const int32_t code = c.read_code[r - c.ra];
      const int n = (int)(c.read_off[r - c.ra + 1] - c.read_off[r - c.ra]);
      if (n <= 0) continue;
      if (bo.long_warp && fp32 && !anchored && !code_general(code) && (code & 512) != 0) {
        emit_long(r);
        continue;
      }
      const bool eligible = pair_reads && !anchored && !code_general(code) && (code & 512) == 0 &&
                            ((bo.pair_mask >> code_R(code)) & 1);
      if (!eligible) { emit(r, -1); continue; }
      const int R = code_R(code);
      if (waiting[R] >= 0) {
        emit(waiting[R], r);
        waiting[R] = -1;
      } else {
        waiting[R] = r;
      }
    }
    for (int k = 0; k <= kMaxR; ++k)
      if (waiting[k] >= 0) emit(waiting[k], -1);
    }
   }
  });
  std::vector<int64_t> cost;
  size_t total = 0;
  for (auto& sl : slices) total += sl.items.size();
  c.items.reserve(total);
  cost.reserve(total);
  for (auto& sl : slices) {
    c.items.insert(c.items.end(), sl.items.begin(), sl.items.end());
    cost.insert(cost.end(), sl.cost.begin(), sl.cost.end());
    c.cells += sl.cells;
    c.shared_cells += sl.shared;
    c.pairs_scored += sl.pairs;
  }
  const int64_t out = region_out_of[ng];
  c.n_out = out;
  if (!plain) order_items(c.items, cost);
  auto mid = std::stable_partition(c.items.begin(), c.items.end(),
                                   [](const WorkItem& w) { return code_paired(w.code); });
  c.n_paired = (int64_t)(mid - c.items.begin());
  c.pair_split = bo.pair_split;
  auto wide = std::stable_partition(c.items.begin(), mid,
                                    [&](const WorkItem& w) { return code_R(w.code) >= bo.pair_split; });
  c.n_paired_wide = (int64_t)(wide - c.items.begin());
  auto lend = std::stable_partition(mid, c.items.end(), [](const WorkItem& w) { return code_long(w.code); });
  c.n_long = (int64_t)(lend - mid);
}

// Pair form: pairs grouped by read (counting sort), each read's haplotypes as
// an indirect list.
struct PairGroups {
  std::vector<int64_t> start;  // per read, n_reads + 1
  std::vector<int64_t> order;  // pair indices grouped by read
};

void group_pairs(const vd_batch* b, PairGroups& pg) {
  pg.start.assign(b->n_reads + 1, 0);
  for (int64_t p = 0; p < b->n_pairs; ++p) ++pg.start[b->pair_read[p] + 1];
  for (int64_t r = 0; r < b->n_reads; ++r) pg.start[r + 1] += pg.start[r];
  std::vector<int64_t> fill(pg.start.begin(), pg.start.end() - 1);
  pg.order.resize(b->n_pairs);
  for (int64_t p = 0; p < b->n_pairs; ++p) pg.order[fill[b->pair_read[p]]++] = p;
}

void build_pair_chunk(const vd_batch* b, const PairGroups& pg, int64_t ra, int64_t rb, const TableSet* ts,
                      bool offsets, bool anchored, HostChunk& c, bool plain = false,
                      const BuildOpts& bo = BuildOpts()) {
  c.ra = ra;
  c.rb = rb;
  c.ha = 0;
  c.hb = b->n_haps;
  finish_chunk_common(c, b, ts, offsets, anchored, bo);
  std::vector<int64_t> cost;
  const int64_t kMaxStream = bo.max_stream;
  for (int64_t r = ra; r < rb; ++r) {
    // the fixed tile of the plain schedule (reads longer than a strip keep the tuned strip height)
    const int32_t rc = c.read_code[r - ra];
    const int32_t code = (plain && (rc & 512) == 0) ? (rc & ~15) | kMaxR : rc;
    const int n = (int)(c.read_off[r - ra + 1] - c.read_off[r - ra]);
    const int R = code_R(code);
    const int n_rows = n + (anchored ? 1 : 0);
    const bool multistrip = plain || n_rows > kStripRows;
    const int64_t rows = n > 0 ? (int64_t)kWarp * R * ((n_rows + kWarp * R - 1) / (kWarp * R)) : 0;
    int64_t list_begin = (int64_t)c.hap_sel.size();
    int64_t stream = 0;
    auto flush = [&]() {
      const int64_t cnt = (int64_t)c.hap_sel.size() - list_begin;
      if (cnt <= 0) return;
      WorkItem w;
      w.read = (int32_t)(r - ra);
      w.nhap = (int32_t)cnt;
      w.hap_begin = list_begin;
      w.out_begin = list_begin;
      w.code = code;
      w.read2 = -1;
        w.out2_begin = 0;
      c.items.push_back(w);
      cost.push_back(rows * (stream + kWarp));
      list_begin = (int64_t)c.hap_sel.size();
      stream = 0;
    };
    for (int64_t k = pg.start[r]; k < pg.start[r + 1]; ++k) {
      const int64_t p = pg.order[k];
      const int64_t h = b->pair_hap[p];
      const int m = (int)(b->hap_off[h + 1] - b->hap_off[h]);
      const int64_t slot = (int64_t)c.out_global.size();
      c.out_global.push_back(p);
      if (n <= 0 || m <= 0) {
        // stays -inf: out_sel keeps no entry for it
        continue;
      }
      if (stream > 0 && (multistrip || stream + m + 1 > kMaxStream)) flush();
      c.hap_sel.push_back((int32_t)h);
      c.out_sel.push_back(slot);
      stream += m + 1;
      c.cells += (int64_t)n * m;
      ++c.pairs_scored;
    }
    flush();
  }
  c.n_out = (int64_t)c.out_global.size();
  if (!plain) order_items(c.items, cost);
}

// Device bytes a chunk needs (inputs, lists, outputs, rescue lists, scratch).
struct Layout {
  size_t o_rb, o_rq, o_roff, o_rcode, o_hb, o_hoff, o_hsel, o_osel, o_hord, o_hshare, o_items, o_out, o_sp1,
      o_sp2, o_cnt, o_scratch, total;
  int64_t scratch_stride;  // double2 records per warp slot
  int64_t warps;
};

Layout layout_for(const HostChunk& c, const vd_batch* b, int64_t warps) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + std::max<size_t>(bytes, 1), 256); return o; };
  const int64_t read_bytes = c.read_off.back();
  const int64_t hap_bytes = c.hap_off.back();
  L.o_rb = take(read_bytes);
  L.o_rq = take(read_bytes);
  L.o_roff = take(c.read_off.size() * sizeof(int64_t));
  L.o_rcode = take(c.read_code.size() * sizeof(int32_t));
  L.o_hb = take(hap_bytes);
  L.o_hoff = take(c.hap_off.size() * sizeof(int64_t));
  L.o_hsel = take(c.hap_sel.size() * sizeof(int32_t));
  L.o_osel = take(c.out_sel.size() * sizeof(int64_t));
  L.o_hord = take(c.hap_order.size() * sizeof(int32_t));
  L.o_hshare = take(c.hap_share.size() * sizeof(int32_t));
  L.o_items = take(c.items.size() * sizeof(WorkItem));
  L.o_out = take((size_t)c.n_out * sizeof(double));
  L.o_sp1 = take((size_t)std::max<int64_t>(1, c.pairs_scored) * sizeof(RescueEntry));
  L.o_sp2 = take((size_t)std::max<int64_t>(1, c.pairs_scored) * sizeof(RescueEntry));
  L.o_cnt = take(16 * sizeof(unsigned long long));
  // the long-read kernel keeps two boundary buffers per warp slot
  L.scratch_stride = c.any_long ? (int64_t)(c.max_hap + 1) * (c.n_long > 0 ? 2 : 1) : 0;
  L.warps = c.any_strip ? warps : std::min<int64_t>(warps, (int64_t)kRobustBlocks * kWarpsPerBlock);
  L.o_scratch = take((size_t)std::max<int64_t>(1, L.scratch_stride) * warps * sizeof(double2));
  L.total = off;
  (void)b;
  return L;
}

// ---- gradient tables ---------------------------------------------------------------

// Derivatives of the folded constants of build_tables with respect to the
// Phred-scale parameters (Qg, Qx, bin offsets).  A quality whose Phred,
// after its offset, is at or below the floor 0 has no offset derivative.
void build_grad_tables(double g, double x, const double* offsets, GradTables* gt, GradScalars* gs) {
  const double L10 = std::log(10.0) / 10.0;
  for (int q = 0; q < 256; ++q) {
    double ph = (double)std::min(q, 60) + (offsets ? offsets[quality_bin((unsigned)q)] : 0.0);
    const bool floor = ph <= 0.0;
    ph = std::max(0.0, ph);
    const double e = std::pow(10.0, -ph / 10.0);
    const double dE = floor ? 0.0 : -L10 * e;  // de / d offset
    const double p1 = 1.0 - e, p0 = e / 3.0;
    gt->bin[q] = quality_bin((unsigned)q);
    if (dE == 0.0) {
      gt->dlnN[q] = gt->dlnmiss[q] = gt->dlnhit[q] = 0.0;
    } else if (p0 > p1) {  // two-sided rows: hit = 3(1-e)/e, miss = 1, N = a e/3
      gt->dlnN[q] = dE / e;
      gt->dlnmiss[q] = 0.0;
      gt->dlnhit[q] = dE * (-1.0 / (1.0 - e) - 1.0 / e);
    } else {               // hit = 1, miss = e/(3(1-e)), N = a (1-e)
      gt->dlnN[q] = -dE / (1.0 - e);
      gt->dlnmiss[q] = dE * (1.0 / e + 1.0 / (1.0 - e));
      gt->dlnhit[q] = 0.0;
    }
  }
  const double a = 1.0 - 2.0 * g, dg = -L10 * g, dx = -L10 * x;
  gs->dlnN_g = (-2.0 / a) * dg;
  gs->dlnK_g = (1.0 / g + 4.0 / a) * dg;
  gs->dlnX_g = (2.0 / a) * dg;
  gs->dlnA_g = (1.0 / g + 2.0 / a) * dg;
  gs->dlnk2_g = (1.0 / g + 2.0 / a) * dg;
  gs->dlng_g = (1.0 / g) * dg;
  gs->dlnK_x = (-1.0 / (1.0 - x)) * dx;
  gs->dlnX_x = (1.0 / x) * dx;
  gs->dlnk2_x = (-1.0 / (1.0 - x)) * dx;
  gs->dx_x = dx;
}

__global__ void fill_kernel(double* p, int64_t n, double v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

}  // namespace

// ---- plan -----------------------------------------------------------------------

struct vd_plan {
  vd_engine* eng = nullptr;
  DevBuf own;              // buffers of a standalone plan
  char* base = nullptr;    // device base of the layout
  Layout L{};
  HostChunk chunk;
  vd_params params{};
  double offsets[4] = {0, 0, 0, 0};
  bool has_offsets = false;
  cudaGraphExec_t graph = nullptr;
  int graph_launches = 0;  // kernels in the captured graph
  // stream and tier events the plan's work is enqueued on (the engine's own,
  // or a pipeline slot's in vd_forward)
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_begin = nullptr, ev_mid = nullptr, ev_end = nullptr;
  cudaStream_t side = nullptr;                        // the long-read kernel's stream
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;  // its fork from and join into `stream`
  int64_t last_rescued1 = 0, last_rescued2 = 0;
};

namespace {

BatchView batch_view(vd_plan* pl) {
  BatchView bv{};
  char* d = pl->base;
  bv.read_bases = (const uint8_t*)(d + pl->L.o_rb);
  bv.read_quals = (const uint8_t*)(d + pl->L.o_rq);
  bv.read_off = (const int64_t*)(d + pl->L.o_roff);
  bv.read_code = (const int32_t*)(d + pl->L.o_rcode);
  bv.hap_bases = (const uint8_t*)(d + pl->L.o_hb);
  bv.hap_off = (const int64_t*)(d + pl->L.o_hoff);
  bv.hap_sel = pl->chunk.hap_sel.empty() && pl->chunk.out_sel.empty() ? nullptr : (const int32_t*)(d + pl->L.o_hsel);
  bv.out_sel = bv.hap_sel ? (const int64_t*)(d + pl->L.o_osel) : nullptr;
  bv.hap_share = pl->chunk.hap_share.empty() ? nullptr : (const int32_t*)(d + pl->L.o_hshare);
  bv.hap_order = pl->chunk.hap_order.empty() ? nullptr : (const int32_t*)(d + pl->L.o_hord);
  bv.out = (double*)(d + pl->L.o_out);
  return bv;
}

int upload_chunk(vd_plan* pl, const vd_batch* b, int64_t* h2d) {
  vd_engine* e = pl->eng;
  HostChunk& c = pl->chunk;
  char* d = pl->base;
  const int64_t read_bytes = c.read_off.back();
  const int64_t hap_bytes = c.hap_off.back();
  int64_t bytes = 0;
  auto put = [&](size_t off, const void* src, size_t n) -> int {
    if (n == 0) return VD_OK;
    VD_CUDA(cudaMemcpyAsync(d + off, src, n, cudaMemcpyHostToDevice, pl->stream));
    bytes += (int64_t)n;
    return VD_OK;
  };
  int rc;
  if ((rc = put(pl->L.o_rb, b->read_bases + b->read_off[c.ra], read_bytes))) return rc;
  if ((rc = put(pl->L.o_rq, b->read_quals + b->read_off[c.ra], read_bytes))) return rc;
  if ((rc = put(pl->L.o_roff, c.read_off.data(), c.read_off.size() * sizeof(int64_t)))) return rc;
  if ((rc = put(pl->L.o_rcode, c.read_code.data(), c.read_code.size() * sizeof(int32_t)))) return rc;
  if ((rc = put(pl->L.o_hb, b->hap_bases + b->hap_off[c.ha], hap_bytes))) return rc;
  if ((rc = put(pl->L.o_hoff, c.hap_off.data(), c.hap_off.size() * sizeof(int64_t)))) return rc;
  if ((rc = put(pl->L.o_hsel, c.hap_sel.data(), c.hap_sel.size() * sizeof(int32_t)))) return rc;
  if ((rc = put(pl->L.o_osel, c.out_sel.data(), c.out_sel.size() * sizeof(int64_t)))) return rc;
  if ((rc = put(pl->L.o_hord, c.hap_order.data(), c.hap_order.size() * sizeof(int32_t)))) return rc;
  if ((rc = put(pl->L.o_hshare, c.hap_share.data(), c.hap_share.size() * sizeof(int32_t)))) return rc;
  if ((rc = put(pl->L.o_items, c.items.data(), c.items.size() * sizeof(WorkItem)))) return rc;
  if (c.n_out > 0) {
    fill_kernel<<<(int)std::min<int64_t>(4096, (c.n_out + 255) / 256), 256, 0, pl->stream>>>(
        (double*)(d + pl->L.o_out), c.n_out, -HUGE_VAL);
    VD_CUDA(cudaGetLastError());
  }
  if (h2d) *h2d += bytes;
  return VD_OK;
}

// Enqueue the three tiers on the engine stream, bracketed by the engine's
// events: ev_begin .. ev_mid is the primary tier, ev_mid .. ev_end the rescue.
int enqueue_tiers(vd_plan* pl, int* launches, bool capturing = false) {
  vd_engine* e = pl->eng;
  char* d = pl->base;
  const Layout& L = pl->L;
  const bool anch = pl->params.anchored != 0;
  const bool f64 = pl->params.precision == VD_PRECISION_FLOAT64;
  unsigned long long* cnt = (unsigned long long*)(d + L.o_cnt);
  // inside a stream capture an event becomes a graph node only when recorded
  // as external; otherwise it would only order the capture
  const unsigned evflags = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  cudaGetLastError();  // launch checks below must see only their own errors
  // cnt[0..2] work heads of tiers 0..2, cnt[3], cnt[4] spill counts, cnt[5] error flag,
  // cnt[6..7] heads of the two-read kernels, cnt[8] spill count of the FP64
  // tier, cnt[9] head of the drift tier (FP32 semiglobal only), cnt[10]
  // head of the long-read kernel, cnt[11..12] its runs of strips and strips
  VD_CUDA(cudaMemsetAsync(cnt, 0, 16 * sizeof(unsigned long long), pl->stream));
  VD_CUDA(cudaEventRecordWithFlags(pl->ev_begin, pl->stream, evflags));
  const BatchView bv = batch_view(pl);
  // device tables by address; the scalars by value from the host copy
  TableSet* dt = (TableSet*)e->dtab.p;
  const TableSet* ht = e->htab;
  QueueView q{};
  q.scratch = d + L.o_scratch;
  q.scratch_stride = L.scratch_stride;
  q.error_flag = (int*)(cnt + 5);
  const int64_t cap = std::max<int64_t>(1, pl->chunk.pairs_scored);
  // tier 0
  q.items = (const WorkItem*)(d + L.o_items);
  q.entries = nullptr;
  q.count = nullptr;
  q.n_items = (long long)pl->chunk.items.size();
  q.head = cnt + 0;
  q.spill = (RescueEntry*)(d + L.o_sp1);
  q.spill_count = cnt + 3;
  q.spill_cap = cap;
  int n = 0;
  if (!pl->chunk.items.empty()) {
    cudaError_t err = cudaSuccess;
    const int64_t np = pl->chunk.n_paired, nw = pl->chunk.n_paired_wide;
    const int64_t nl = pl->chunk.n_long;
    q.static_order = pl->params.schedule == VD_SCHEDULE_PLAIN ? 1 : 0;
    if (nl > 0) {
      // long reads, up to kLongGroupMax haplotypes per warp item, launched
      // first on the side stream: the kernels below take the SMs its blocks
      // leave as its queue runs dry, so they fill its tail; its failures join
      // the spill list
      VD_CUDA(cudaEventRecord(pl->ev_fork, pl->stream));
      VD_CUDA(cudaStreamWaitEvent(pl->side, pl->ev_fork, 0));
      QueueView ql = q;
      ql.items = (const WorkItem*)(d + L.o_items) + np;
      ql.n_items = nl;
      ql.head = cnt + 10;
      ql.strip_runs = cnt + 11;  // cnt[11] runs of strips, cnt[12] strips
      const int R = pl->chunk.long_R;
      const bool blk = pl->chunk.long_block;
      err = launch_long_f32(R, blk, bv, ql, &dt->f32, ht->s32d, e->grid_long[blk ? 1 : 0][R == 8 ? 1 : 0], pl->side);
      if (err != cudaSuccess) return cuda_fail(err, "long-read tier launch");
      ++n;
      VD_CUDA(cudaEventRecord(pl->ev_join, pl->side));
    }
    // two-read items, on their own kernels (FP32 semiglobal only): 6-8 rows
    // per lane, then up to 5
    for (int k = 0; k < 2; ++k) {
      const int64_t lo = k ? nw : 0, hi = k ? np : nw;
      if (hi <= lo) continue;
      QueueView qp = q;
      qp.items = (const WorkItem*)(d + L.o_items) + lo;
      qp.n_items = hi - lo;
      qp.head = cnt + 6 + k;
      const int split = pl->chunk.pair_split;
      err = launch_pair_f32(k == 0, split, bv, qp, &dt->f32, ht->s32, e->grid_pair[split == 7][k == 0 ? 1 : 0],
                            pl->stream);
      if (err != cudaSuccess) return cuda_fail(err, "two-read tier launch");
      ++n;
    }
    q.items = (const WorkItem*)(d + L.o_items) + np + nl;
    q.n_items = (long long)(pl->chunk.items.size() - np - nl);
    if (q.n_items > 0) {
      err = f64 ? launch_f64(anch, bv, q, &dt->f64, ht->s64, 1, e->grid[1][anch], pl->stream)
                : launch_f32(anch, bv, q, &dt->f32, ht->s32, 0, e->grid[0][anch], pl->stream);
      if (err != cudaSuccess) return cuda_fail(err, "primary tier launch");
      ++n;
    }
    if (nl > 0) VD_CUDA(cudaStreamWaitEvent(pl->stream, pl->ev_join, 0));
    VD_CUDA(cudaEventRecordWithFlags(pl->ev_mid, pl->stream, evflags));
    BatchView rv = bv;
    rv.hap_sel = nullptr;
    rv.out_sel = nullptr;
    q.static_order = 0;  // the rescue tiers always run on the shared counter
    // the lists: tier 0 spills into sp1; with the drift tier (FP32
    // semiglobal) the chain is sp1 -> drift -> sp2 -> FP64 -> sp1 (cnt[8]) ->
    // robust, otherwise sp1 -> FP64 -> sp2 -> robust
    const bool drift = !f64 && !anch;
    QueueView q1 = q;
    if (drift) {
      QueueView qd = q;
      qd.items = nullptr;
      qd.entries = (const RescueEntry*)(d + L.o_sp1);
      qd.count = cnt + 3;
      qd.n_items = cap;
      qd.head = cnt + 9;
      qd.spill = (RescueEntry*)(d + L.o_sp2);
      qd.spill_count = cnt + 4;
      qd.scratch_stride = 2 * L.scratch_stride;  // two float2 boundaries in each warp's double2 slot
      err = launch_drift_f32(rv, qd, &dt->f32, ht->s32d, e->grid_drift, pl->stream);
      if (err != cudaSuccess) return cuda_fail(err, "drift tier launch");
      ++n;
    }
    if (!f64) {
      // tier 1: FP64 wavefront over the FP32 spills
      q1.items = nullptr;
      q1.entries = (const RescueEntry*)(d + (drift ? L.o_sp2 : L.o_sp1));
      q1.count = cnt + (drift ? 4 : 3);
      q1.n_items = cap;
      q1.head = cnt + 1;
      q1.spill = (RescueEntry*)(d + (drift ? L.o_sp1 : L.o_sp2));
      q1.spill_count = cnt + (drift ? 8 : 4);
      err = launch_f64(anch, rv, q1, &dt->f64, ht->s64, 1, e->grid[1][anch], pl->stream);
      if (err != cudaSuccess) return cuda_fail(err, "rescue tier launch");
      ++n;
    }
    // tier 2: FP64 32-row strips over what the FP64 wavefront spilled
    QueueView q2 = q;
    q2.items = nullptr;
    q2.entries = (const RescueEntry*)(d + ((f64 || drift) ? L.o_sp1 : L.o_sp2));
    q2.count = cnt + (f64 ? 3 : drift ? 8 : 4);
    q2.n_items = cap;
    q2.head = cnt + 2;
    q2.spill = nullptr;
    q2.spill_count = nullptr;
    q2.spill_cap = 0;
    const int robust_grid = pl->chunk.any_strip ? e->grid[1][anch] : std::min(e->grid[1][anch], kRobustBlocks);
    err = launch_f64(anch, rv, q2, &dt->f64, ht->s64, 2, robust_grid, pl->stream);
    if (err != cudaSuccess) return cuda_fail(err, "robust tier launch");
    ++n;
  } else {
    VD_CUDA(cudaEventRecordWithFlags(pl->ev_mid, pl->stream, evflags));
  }
  VD_CUDA(cudaEventRecordWithFlags(pl->ev_end, pl->stream, evflags));
  if (launches) *launches = n;
  return VD_OK;
}

int tier_times(const vd_plan* pl, double* total, double* primary, double* rescue) {
  float a = 0.f, b = 0.f;
  VD_CUDA(cudaEventElapsedTime(&a, pl->ev_begin, pl->ev_mid));
  VD_CUDA(cudaEventElapsedTime(&b, pl->ev_mid, pl->ev_end));
  *primary += a;
  *rescue += b;
  *total += a + b;
  return VD_OK;
}

int enqueue_counter_read(vd_plan* pl, unsigned long long* host) {
  VD_CUDA(cudaMemcpyAsync(host, pl->base + pl->L.o_cnt, 13 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                          pl->stream));
  return VD_OK;
}

// after the plan's stream completed: pairs rescued by the drift tier (r0),
// recomputed in the FP64 wavefront (r1) and in FP64 32-row strips (r2)
int check_counters(const vd_plan* pl, const unsigned long long* h, int64_t* r0, int64_t* r1, int64_t* r2,
                   int64_t* runs = nullptr, int64_t* strips = nullptr) {
  if (h[5]) return fail(VD_EOVERFLOW, "rescue list overflow");
  if (runs) *runs = (int64_t)h[11];
  if (strips) *strips = (int64_t)h[12];
  const bool f64 = pl->params.precision == VD_PRECISION_FLOAT64;
  const bool drift = !f64 && !pl->params.anchored;
  *r0 = drift ? (int64_t)(h[3] - h[4]) : 0;
  *r1 = f64 ? 0 : (int64_t)(drift ? h[4] : h[3]);
  *r2 = (int64_t)(f64 ? h[3] : drift ? h[8] : h[4]);
  return VD_OK;
}

int read_counters(vd_plan* pl, int64_t* r0, int64_t* r1, int64_t* r2, int64_t* runs, int64_t* strips) {
  unsigned long long h[13];
  int rc = enqueue_counter_read(pl, h);
  if (rc) return rc;
  VD_CUDA(cudaStreamSynchronize(pl->stream));
  return check_counters(pl, h, r0, r1, r2, runs, strips);
}

int init_engine_grids(vd_engine* e) {
  for (int f = 0; f < 2; ++f)
    for (int a = 0; a < 2; ++a) {
      int bps = 0;
      cudaError_t err = f ? occupancy_f64(a != 0, &bps) : occupancy_f32(a != 0, &bps);
      if (err != cudaSuccess) return cuda_fail(err, "occupancy query");
      e->grid[f][a] = std::max(1, bps) * e->sm_count;
    }
  int bps = 0;
  cudaError_t err = cudaSuccess;
  for (int sp = 0; sp < 2; ++sp)
    for (int wide = 0; wide < 2; ++wide) {
      bps = 0;
      err = occupancy_pair_f32(wide != 0, sp ? 7 : 6, &bps);
      if (err != cudaSuccess) return cuda_fail(err, "occupancy query");
      e->grid_pair[sp][wide] = std::max(1, bps) * e->sm_count;
    }
  bps = 0;
  err = occupancy_drift_f32(&bps);
  if (err != cudaSuccess) return cuda_fail(err, "occupancy query");
  // its warps index the strip scratch, which is sized by the largest grid
  e->grid_drift = std::min(std::max(1, bps) * e->sm_count, e->grid[0][0]);
  for (int blk = 0; blk < 2; ++blk)
    for (int k = 0; k < 2; ++k) {
      bps = 0;
      err = occupancy_long_f32(k ? 8 : 4, blk != 0, &bps);
      if (err != cudaSuccess) return cuda_fail(err, "occupancy query");
      e->grid_long[blk][k] = std::min(std::max(1, bps) * e->sm_count, e->grid[0][0]);
    }
  for (int f = 0; f < 2; ++f) {
    bps = 0;
    err = occupancy_grad(f != 0, &bps);
    if (err != cudaSuccess) return cuda_fail(err, "occupancy query");
    e->grid_grad[f] = std::max(1, bps) * e->sm_count;
  }
  return VD_OK;
}

int64_t max_grid_warps(const vd_engine* e) {
  int g = 0;
  for (int f = 0; f < 2; ++f) for (int a = 0; a < 2; ++a) g = std::max(g, e->grid[f][a]);
  return (int64_t)g * kWarpsPerBlock;
}

std::mutex g_default_mu;
vd_engine* g_default = nullptr;

int default_engine(vd_engine** out) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default) {
    const char* dev = std::getenv("VARDEPTH_CUDA_DEVICE");
    const char* mb = std::getenv("VARDEPTH_CUDA_MEMORY_MB");
    int rc = vd_engine_create(dev ? std::atoi(dev) : 0, mb ? std::atoll(mb) : 4096, &g_default);
    if (rc) return rc;
  }
  *out = g_default;
  return VD_OK;
}

int default_precision() {
  const char* p = std::getenv("VARDEPTH_CUDA_PRECISION");
  if (p && std::strcmp(p, "float64") == 0) return VD_PRECISION_FLOAT64;
  return VD_PRECISION_MIXED;
}

}  // namespace

namespace vd {
// Records the calling thread's error for vd_last_error (used by the other
// translation units of the library) and returns the code.
int report_error(int code, const char* msg) { return fail(code, msg); }

// The model tables of one (gap, ext, offsets) setting for callers outside this
// file (the no-allocation entry point builds them into its own buffers).
void build_model_tables(double gap, double ext, const double* offsets, Tables<float>* f32, Tables<double>* f64,
                        Scalars<float>* s32, Scalars<double>* s64) {
  static TableSet ts;  // 40 KB; callers serialise on their own lock
  build_tables(gap, ext, offsets, &ts);
  *f32 = ts.f32;
  *f64 = ts.f64;
  *s32 = ts.s32;
  *s64 = ts.s64;
}
}  // namespace vd

extern "C" {

const char* vd_last_error(void) { return g_last_error.c_str(); }

const char* vd_version(void) { return "vardepth-pairhmm-b200 0.1 sm_100a"; }

int vd_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n;
}

int vd_engine_create(int device, int64_t memory_mb, vd_engine** out) {
  if (!out) return fail(VD_EINVAL, "out is NULL");
  *out = nullptr;
  if (memory_mb < 8) return fail(VD_EINVAL, "CUDA workspace budget must be at least 8 MiB");
  int count = 0;
  cudaError_t err = cudaGetDeviceCount(&count);
  if (err != cudaSuccess || count <= 0) {
    cudaGetLastError();
    return fail(VD_ENODEV, "CUDA PairHMM requires an accessible NVIDIA GPU");
  }
  if (device < 0 || device >= count) return fail(VD_ENODEV, "CUDA device index out of range");
  DeviceGuard guard(device);
  cudaDeviceProp prop;
  VD_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(VD_ENODEV, "this library is built for sm_100a (B200) only");
  vd_engine* e = new vd_engine();
  e->device = device;
  e->sm_count = prop.multiProcessorCount;
  e->cc_major = prop.major;
  e->cc_minor = prop.minor;
  std::snprintf(e->name, sizeof(e->name), "%s", prop.name);
  e->budget = (size_t)memory_mb << 20;
  int rc = VD_OK;
  if ((err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (err = cudaEventCreate(&e->ev_begin)) != cudaSuccess || (err = cudaEventCreate(&e->ev_mid)) != cudaSuccess ||
      (err = cudaEventCreate(&e->ev_end)) != cudaSuccess ||
      (err = cudaStreamCreateWithFlags(&e->side, cudaStreamNonBlocking)) != cudaSuccess ||
      (err = cudaEventCreateWithFlags(&e->ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaEventCreateWithFlags(&e->ev_join, cudaEventDisableTiming)) != cudaSuccess ||
      (err = cudaMallocHost((void**)&e->htab, sizeof(TableSet))) != cudaSuccess) {
    rc = cuda_fail(err, "engine setup");
  }
  for (int k = 0; k < 2 && !rc; ++k) {
    vd_engine::Slot& sl = e->slots[k];
    if ((err = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (err = cudaEventCreate(&sl.ev[0])) != cudaSuccess || (err = cudaEventCreate(&sl.ev[1])) != cudaSuccess ||
        (err = cudaEventCreate(&sl.ev[2])) != cudaSuccess ||
        (err = cudaStreamCreateWithFlags(&sl.side, cudaStreamNonBlocking)) != cudaSuccess ||
        (err = cudaEventCreateWithFlags(&sl.fork, cudaEventDisableTiming)) != cudaSuccess ||
        (err = cudaEventCreateWithFlags(&sl.join, cudaEventDisableTiming)) != cudaSuccess ||
        (err = cudaMallocHost((void**)&sl.hcnt, 16 * sizeof(unsigned long long))) != cudaSuccess)
      rc = cuda_fail(err, "engine pipeline setup");
  }
  if (!rc) rc = init_engine_grids(e);
  if (rc) { vd_engine_destroy(e); return rc; }
  *out = e;
  return VD_OK;
}

int vd_engine_destroy(vd_engine* e) {
  if (!e) return VD_OK;
  {
    DeviceGuard guard(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    if (e->side) cudaStreamSynchronize(e->side);
    // plans still alive become empty shells; vd_plan_destroy frees the shell
    for (vd_plan* pl : e->plans) {
      if (pl->graph) cudaGraphExecDestroy(pl->graph);
      pl->graph = nullptr;
      pl->own.release();
      pl->base = nullptr;
      pl->eng = nullptr;
    }
    e->plans.clear();
    for (vd_engine::Slot& sl : e->slots) {
      if (sl.stream) cudaStreamSynchronize(sl.stream);
      if (sl.side) cudaStreamSynchronize(sl.side);
      delete sl.pl;
      sl.pl = nullptr;
      sl.arena.release();
      for (cudaEvent_t& ev : sl.ev) if (ev) cudaEventDestroy(ev);
      if (sl.fork) cudaEventDestroy(sl.fork);
      if (sl.join) cudaEventDestroy(sl.join);
      if (sl.hcnt) cudaFreeHost(sl.hcnt);
      if (sl.side) cudaStreamDestroy(sl.side);
      if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    e->arena.release();
    e->grad_arena.release();
    e->geno_arena.release();
    e->dtab.release();
    if (e->htab) cudaFreeHost(e->htab);
    if (e->ev_begin) cudaEventDestroy(e->ev_begin);
    if (e->ev_mid) cudaEventDestroy(e->ev_mid);
    if (e->ev_end) cudaEventDestroy(e->ev_end);
    if (e->ev_fork) cudaEventDestroy(e->ev_fork);
    if (e->ev_join) cudaEventDestroy(e->ev_join);
    if (e->side) cudaStreamDestroy(e->side);
    if (e->stream) cudaStreamDestroy(e->stream);
  }
  if (e == g_default) g_default = nullptr;
  delete e;
  return VD_OK;
}

int vd_engine_info(const vd_engine* e, char* name, int name_len, int* major, int* minor, int* sm_count) {
  if (!e) return fail(VD_EINVAL, "engine is NULL");
  if (name && name_len > 0) std::snprintf(name, (size_t)name_len, "%s", e->name);
  if (major) *major = e->cc_major;
  if (minor) *minor = e->cc_minor;
  if (sm_count) *sm_count = e->sm_count;
  return VD_OK;
}

int vd_engine_set_tuning(vd_engine* e, const vd_tuning* t) {
  if (!e || !t) return fail(VD_EINVAL, "engine or tuning is NULL");
  if (t->long_read_rows != 64 && t->long_read_rows != 128 && t->long_read_rows != 256)
    return fail(VD_EINVAL, "long_read_rows must be 64, 128 or 256");
  if (t->pair_mask & ~0x1fe) return fail(VD_EINVAL, "pair_mask holds bits 1..8 only");
  if (t->max_item_columns < 0) return fail(VD_EINVAL, "max_item_columns must be >= 0");
  if (t->pipeline_gcells < 0) return fail(VD_EINVAL, "pipeline_gcells must be >= 0");
  if (t->long_mode != VD_LONG_WARP && t->long_mode != VD_LONG_SINGLE && t->long_mode != VD_LONG_BLOCK)
    return fail(VD_EINVAL, "long_mode must be VD_LONG_WARP, VD_LONG_SINGLE or VD_LONG_BLOCK");
  if (t->pair_split != 0 && t->pair_split != 6 && t->pair_split != 7)
    return fail(VD_EINVAL, "pair_split must be 6 or 7 (0 = 6)");
  if (t->long_group < 0 || t->long_group > kLongGroupMax)
    return fail(VD_EINVAL, "long_group must be 1..8 (0 = 8)");
  if (t->reserved[0]) return fail(VD_EINVAL, "reserved fields must be zero");
  std::lock_guard<std::mutex> lk(e->mu);
  e->tuning = *t;
  return VD_OK;
}

int vd_engine_get_tuning(const vd_engine* e, vd_tuning* t) {
  if (!e || !t) return fail(VD_EINVAL, "engine or tuning is NULL");
  *t = e->tuning;
  return VD_OK;
}

int64_t vd_batch_outputs(const vd_batch* b) {
  if (validate_batch(b)) return -1;
  return batch_outputs(b);
}

int vd_prefix_plan(const unsigned char* hap_bases, const int64_t* hap_off, int64_t n_haps, int32_t* order,
                   int32_t* share) {
  if (n_haps < 0 || (n_haps > 0 && (!hap_off || !order || !share))) return fail(VD_EINVAL, "NULL argument");
  if (n_haps == 0) return VD_OK;
  if (n_haps > INT32_MAX || !offsets_ok(hap_off, n_haps))
    return fail(VD_EINVAL, "haplotype offsets must be non-decreasing (lengths <= 2^28)");
  if (hap_off[n_haps] > hap_off[0] && !hap_bases) return fail(VD_EINVAL, "haplotype buffer is NULL");
  vd_batch b{};
  b.hap_bases = hap_bases;
  b.hap_off = hap_off;
  b.n_haps = n_haps;
  region_order_and_shares(&b, 0, n_haps, 0, order, share);
  return VD_OK;
}

int vd_forward(vd_engine* e, const vd_batch* b, const vd_params* p, double* out, vd_stats* st) {
  const double t0 = now_ms();
  if (!e) return fail(VD_EINVAL, "engine is NULL");
  int rc = validate_params(p);
  if (!rc) rc = validate_batch(b);
  if (rc) return rc;
  const int64_t n_out = batch_outputs(b);
  if (n_out > 0 && !out) return fail(VD_EINVAL, "out is NULL");
  std::lock_guard<std::mutex> lk(e->mu);
  DeviceGuard guard(e->device);
  vd_stats s{};
  s.pairs = n_out;
  if ((rc = ensure_tables(e, p))) return rc;
  const bool offsets = p->quality_offsets != nullptr;
  const int64_t warps = max_grid_warps(e);

  // chunk boundaries: regions (region form) or reads (pair form)
  PairGroups pg;
  const bool pair_form = b->pair_read != nullptr;
  if (pair_form) group_pairs(b, pg);
  const int64_t units = pair_form ? b->n_reads : b->n_regions;
  // bytes per unit, estimated from inputs; a chunk grows until the estimate
  // reaches the budget (accelerator.py:118-121 semantics)
  auto unit_bytes = [&](int64_t u) -> int64_t {
    if (pair_form) {
      const int64_t n = b->read_off[u + 1] - b->read_off[u];
      const int64_t np = pg.start[u + 1] - pg.start[u];
      return 2 * n + 64 + np * (4 + 8 + 8 + 32) + 64;
    }
    const int64_t r0 = b->region_read_off[u], r1 = b->region_read_off[u + 1];
    const int64_t h0 = b->region_hap_off[u], h1 = b->region_hap_off[u + 1];
    const int64_t np = (r1 - r0) * (h1 - h0);
    return 2 * (b->read_off[r1] - b->read_off[r0]) + (r1 - r0) * 64 + (b->hap_off[h1] - b->hap_off[h0]) +
           (h1 - h0) * 8 + np * (8 + 32);
  };
  // DP cells per unit: large batches are cut into several chunks so that the
  // host work of one chunk overlaps the kernels of the previous one
  auto unit_cells = [&](int64_t u) -> int64_t {
    if (pair_form) return (b->read_off[u + 1] - b->read_off[u]) * 512 * (pg.start[u + 1] - pg.start[u]);
    const int64_t r0 = b->region_read_off[u], r1 = b->region_read_off[u + 1];
    const int64_t h0 = b->region_hap_off[u], h1 = b->region_hap_off[u + 1];
    return (b->read_off[r1] - b->read_off[r0]) * (b->hap_off[h1] - b->hap_off[h0]);
  };
  int64_t total_cells = 0;
  for (int64_t u = 0; u < units; ++u) total_cells += unit_cells(u);
  // warp items of the long-read kernel (reads longer than a strip, up to
  // long_group haplotypes each)
  const BuildOpts lbo = build_opts(e);
  int64_t long_items = 0;
  if (lbo.long_warp && !lbo.long_block && p->precision != VD_PRECISION_FLOAT64 && !p->anchored) {
    auto long_reads = [&](int64_t r0, int64_t r1) {
      int64_t k = 0;
      for (int64_t r = r0; r < r1; ++r) k += (b->read_off[r + 1] - b->read_off[r]) > kStripRows;
      return k;
    };
    for (int64_t u = 0; u < units; ++u) {
      const int64_t nh = pair_form ? pg.start[u + 1] - pg.start[u] : b->region_hap_off[u + 1] - b->region_hap_off[u];
      const int64_t nl = pair_form ? long_reads(u, u + 1) : long_reads(b->region_read_off[u], b->region_read_off[u + 1]);
      long_items += nl * ((nh + lbo.long_group - 1) / lbo.long_group);
    }
  }
  // The first chunk is a quarter of the others: its host work and upload are
  // the only ones not hidden behind kernels.  Chunks run one after another on
  // the device, so each keeps at least kLongItemsPerWarp long-read items per
  // warp (a chunk's last long items would otherwise run alone on the GPU).
  constexpr int64_t kLongItemsPerWarp = 8;
  const int64_t pipeline_cells = (int64_t)(e->tuning.pipeline_gcells > 0 ? e->tuning.pipeline_gcells : 300) * 1'000'000'000LL;
  int64_t n_pipe = std::max<int64_t>(1, std::min<int64_t>(8, total_cells / pipeline_cells));
  if (long_items > 0) {
    const int64_t long_warps = (int64_t)e->grid_long[0][lbo.long_R == 8 ? 1 : 0] * kWarpsPerBlock;
    n_pipe = std::max<int64_t>(1, std::min<int64_t>(n_pipe, long_items / (kLongItemsPerWarp * std::max<int64_t>(1, long_warps))));
  }
  const int64_t chunk_cells = n_pipe > 1 ? (total_cells + n_pipe - 1) / n_pipe : INT64_MAX;

  int64_t fixed = pair_form ? (b->hap_off[b->n_haps] - b->hap_off[0]) + 8 * b->n_haps : 0;
  int64_t max_hap = 0, max_read = 0;
  for (int64_t h = 0; h < b->n_haps; ++h) max_hap = std::max<int64_t>(max_hap, b->hap_off[h + 1] - b->hap_off[h]);
  for (int64_t r = 0; r < b->n_reads; ++r) max_read = std::max<int64_t>(max_read, b->read_off[r + 1] - b->read_off[r]);
  const int64_t scratch_warps = max_read + p->anchored > kStripRows ? warps : std::min<int64_t>(warps, (int64_t)kRobustBlocks * kWarpsPerBlock);
  // (two boundary buffers per warp slot when the long-read kernel runs)
  fixed += (max_hap + 1) * scratch_warps * (int64_t)sizeof(double2) * (max_read > kStripRows ? 2 : 1) + 64 * 1024;
  const int64_t budget = (int64_t)e->budget;

  // results of the chunk in a slot, once its stream has completed
  auto finish = [&](vd_engine::Slot& sl) -> int {
    if (!sl.busy) return VD_OK;
    sl.busy = false;
    VD_CUDA(cudaStreamSynchronize(sl.stream));
    vd_plan& pl = *sl.pl;
    int64_t r0 = 0, r1 = 0, r2 = 0, lr = 0, ls = 0;
    int r = check_counters(&pl, sl.hcnt, &r0, &r1, &r2, &lr, &ls);
    if (r) return r;
    if ((r = tier_times(&pl, &s.kernel_ms, &s.primary_ms, &s.rescue_ms))) return r;
    s.long_strip_runs += lr;
    s.long_strips += ls;
    s.rescued_fp32 += r0;
    s.rescued_fp64 += r1;
    s.rescued_robust += r2;
    const HostChunk& c = pl.chunk;
    if (pair_form) for (int64_t k = 0; k < c.n_out; ++k) out[c.out_global[k]] = sl.stage[k];
    return VD_OK;
  };

  int64_t u = 0, chunk_index = 0;
  // The kernels of a chunk wait for all kernels of the previous chunk (its
  // copies do not): FP32 kernels of two chunks sharing the SMs run different
  // variants side by side and thrash the instruction cache, and rescue tiers
  // queued behind the next chunk's persistent kernels hold back their chunk's
  // completion, and with it the host's next build, until that chunk's
  // primary tier ends.
  cudaEvent_t prev_end = nullptr;
  while (u < units) {
    int64_t u_end = u, bytes = fixed, cells = 0;
    while (u_end < units) {
      const int64_t ub = unit_bytes(u_end);
      if (u_end > u && (bytes + ub > budget || cells >= (chunk_index == 0 ? chunk_cells / 4 : chunk_cells))) break;
      bytes += ub;
      cells += unit_cells(u_end);
      ++u_end;
    }
    if (bytes > budget) return fail(VD_ENOMEM, "One pair exceeds CUDA workspace budget");
    vd_engine::Slot& sl = e->slots[chunk_index & 1];
    if ((rc = finish(sl))) return rc;  // the slot's previous chunk
    if (!sl.pl) sl.pl = new vd_plan();
    vd_plan& pl = *sl.pl;
    pl.chunk = HostChunk();
    pl.eng = e;
    pl.params = *p;
    pl.stream = sl.stream;
    pl.ev_begin = sl.ev[0];
    pl.ev_mid = sl.ev[1];
    pl.ev_end = sl.ev[2];
    pl.side = sl.side;
    pl.ev_fork = sl.fork;
    pl.ev_join = sl.join;
    const double th = now_ms();
    const bool plain = p->schedule == VD_SCHEDULE_PLAIN;
    const BuildOpts bo = build_opts(e);
    if (pair_form) build_pair_chunk(b, pg, u, u_end, e->htab, offsets, p->anchored != 0, pl.chunk, plain, bo);
    else build_region_chunk(b, u, u_end, e->htab, offsets, p->anchored != 0, p->precision == VD_PRECISION_MIXED,
                            pl.chunk, plain, bo);
    HostChunk& c = pl.chunk;
    pl.L = layout_for(c, b, warps);
    s.host_ms += now_ms() - th;
    if ((rc = sl.arena.reserve(pl.L.total))) return rc;
    pl.base = (char*)sl.arena.p;
    s.live_bytes = std::max<int64_t>(s.live_bytes, (int64_t)(e->slots[0].arena.bytes + e->slots[1].arena.bytes));
    if ((rc = upload_chunk(&pl, b, &s.h2d_bytes))) return rc;
    if (prev_end) VD_CUDA(cudaStreamWaitEvent(pl.stream, prev_end, 0));
    int launches = 0;
    if ((rc = enqueue_tiers(&pl, &launches))) return rc;
    prev_end = pl.ev_end;
    s.kernel_launches += launches + (c.n_out > 0 ? 1 : 0);  // the -inf fill of the upload
    const double* dout = (const double*)(pl.base + pl.L.o_out);
    if (c.n_out > 0) {
      if (pair_form) {
        sl.stage.resize((size_t)c.n_out);
        VD_CUDA(cudaMemcpyAsync(sl.stage.data(), dout, (size_t)c.n_out * sizeof(double), cudaMemcpyDeviceToHost, sl.stream));
      } else {
        VD_CUDA(cudaMemcpyAsync(out + c.out_begin, dout, (size_t)c.n_out * sizeof(double), cudaMemcpyDeviceToHost, sl.stream));
      }
      s.d2h_bytes += c.n_out * (int64_t)sizeof(double);
    }
    if ((rc = enqueue_counter_read(&pl, sl.hcnt))) return rc;
    sl.busy = true;
    s.dp_cells += c.cells;
    s.shared_cells += c.shared_cells;
    s.work_items += (int64_t)c.items.size();
    ++s.batches;
    ++chunk_index;
    u = u_end;
  }
  // drain in submission order
  if ((rc = finish(e->slots[chunk_index & 1]))) return rc;
  if ((rc = finish(e->slots[(chunk_index + 1) & 1]))) return rc;
  s.total_ms = now_ms() - t0;
  if (st) *st = s;
  return VD_OK;
}

int vd_plan_create(vd_engine* e, const vd_batch* b, const vd_params* p, vd_plan** out) {
  if (!e || !out) return fail(VD_EINVAL, "engine or out is NULL");
  *out = nullptr;
  int rc = validate_params(p);
  if (!rc) rc = validate_batch(b);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(e->mu);
  DeviceGuard guard(e->device);
  if ((rc = ensure_tables(e, p))) return rc;
  vd_plan* pl = new vd_plan();
  pl->eng = e;
  pl->params = *p;
  pl->stream = e->stream;
  pl->ev_begin = e->ev_begin;
  pl->ev_mid = e->ev_mid;
  pl->ev_end = e->ev_end;
  pl->side = e->side;
  pl->ev_fork = e->ev_fork;
  pl->ev_join = e->ev_join;
  if (p->quality_offsets) {
    pl->has_offsets = true;
    for (int i = 0; i < 4; ++i) pl->offsets[i] = p->quality_offsets[i];
    pl->params.quality_offsets = pl->offsets;
  }
  const bool offsets = p->quality_offsets != nullptr;
  const bool plain = p->schedule == VD_SCHEDULE_PLAIN;
  const BuildOpts bo = build_opts(e);
  if (b->pair_read) {
    PairGroups pg;
    group_pairs(b, pg);
    build_pair_chunk(b, pg, 0, b->n_reads, e->htab, offsets, p->anchored != 0, pl->chunk, plain, bo);
  } else {
    build_region_chunk(b, 0, b->n_regions, e->htab, offsets, p->anchored != 0, p->precision == VD_PRECISION_MIXED,
                       pl->chunk, plain, bo);
  }
  pl->L = layout_for(pl->chunk, b, max_grid_warps(e));
  if ((rc = pl->own.reserve(pl->L.total))) { delete pl; return rc; }
  pl->base = (char*)pl->own.p;
  if ((rc = upload_chunk(pl, b, nullptr))) { delete pl; return rc; }
  cudaError_t err = cudaStreamSynchronize(e->stream);
  if (err != cudaSuccess) { delete pl; return cuda_fail(err, "plan upload"); }
  // the input buffers of the batch are no longer needed on the host side
  e->plans.insert(pl);
  *out = pl;
  return VD_OK;
}

int vd_plan_run(vd_plan* pl, vd_stats* st) {
  if (!pl) return fail(VD_EINVAL, "plan is NULL");
  if (!pl->eng) return fail(VD_EINVAL, "the plan's engine was destroyed");
  vd_engine* e = pl->eng;
  const double t0 = now_ms();
  std::lock_guard<std::mutex> lk(e->mu);
  DeviceGuard guard(e->device);
  int rc;
  if ((rc = ensure_tables(e, &pl->params))) return rc;
  int launches = 0;
  if (!pl->graph) {
    cudaGraph_t g = nullptr;
    VD_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    rc = enqueue_tiers(pl, &launches, true);
    cudaError_t err = cudaStreamEndCapture(e->stream, &g);
    if (rc) { if (g) cudaGraphDestroy(g); return rc; }
    if (err != cudaSuccess) return cuda_fail(err, "graph capture");
    pl->graph_launches = launches;
    err = cudaGraphInstantiate(&pl->graph, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) { pl->graph = nullptr; return cuda_fail(err, "graph instantiate"); }
  } else {
    launches = pl->graph_launches;
  }
  VD_CUDA(cudaGraphLaunch(pl->graph, e->stream));
  int64_t r0 = 0, r1 = 0, r2 = 0, lr = 0, ls = 0;
  if ((rc = read_counters(pl, &r0, &r1, &r2, &lr, &ls))) return rc;
  double ms = 0.0, pms = 0.0, rms = 0.0;
  if ((rc = tier_times(pl, &ms, &pms, &rms))) return rc;
  pl->last_rescued1 = r1;
  pl->last_rescued2 = r2;
  if (st) {
    vd_stats s{};
    s.pairs = pl->chunk.n_out;
    s.dp_cells = pl->chunk.cells;
    s.shared_cells = pl->chunk.shared_cells;
    s.work_items = (int64_t)pl->chunk.items.size();
    s.batches = 1;
    s.rescued_fp32 = r0;
    s.rescued_fp64 = r1;
    s.rescued_robust = r2;
    s.long_strip_runs = lr;
    s.long_strips = ls;
    s.kernel_launches = launches;
    s.kernel_ms = ms;
    s.primary_ms = pms;
    s.rescue_ms = rms;
    s.total_ms = now_ms() - t0;
    s.live_bytes = (int64_t)pl->L.total;
    *st = s;
  }
  return VD_OK;
}

int vd_plan_fetch(vd_plan* pl, double* out) {
  if (!pl) return fail(VD_EINVAL, "plan is NULL");
  if (!pl->eng) return fail(VD_EINVAL, "the plan's engine was destroyed");
  vd_engine* e = pl->eng;
  const HostChunk& c = pl->chunk;
  if (c.n_out > 0 && !out) return fail(VD_EINVAL, "out is NULL");
  std::lock_guard<std::mutex> lk(e->mu);
  DeviceGuard guard(e->device);
  const double* dout = (const double*)(pl->base + pl->L.o_out);
  if (c.n_out == 0) return VD_OK;
  if (c.out_global.empty()) {
    VD_CUDA(cudaMemcpyAsync(out, dout, (size_t)c.n_out * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    VD_CUDA(cudaStreamSynchronize(e->stream));
  } else {
    std::vector<double> tmp((size_t)c.n_out);
    VD_CUDA(cudaMemcpyAsync(tmp.data(), dout, (size_t)c.n_out * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    VD_CUDA(cudaStreamSynchronize(e->stream));
    for (int64_t k = 0; k < c.n_out; ++k) out[c.out_global[k]] = tmp[k];
  }
  return VD_OK;
}

int vd_plan_destroy(vd_plan* pl) {
  if (!pl) return VD_OK;
  if (vd_engine* e = pl->eng) {
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard guard(e->device);
    cudaStreamSynchronize(e->stream);
    if (pl->graph) cudaGraphExecDestroy(pl->graph);
    pl->graph = nullptr;
    pl->own.release();
    e->plans.erase(pl);
  }
  delete pl;
  return VD_OK;
}

// ---- gradient -----------------------------------------------------------------------

int vd_forward_backward(vd_engine* e, const vd_batch* b, const vd_params* p, int checkpoint, double* out_ln,
                        double* out_jac, vd_grad_stats* st) {
  const double t0 = now_ms();
  if (!e) return fail(VD_EINVAL, "engine is NULL");
  int rc = validate_params(p);
  if (!rc) rc = validate_batch(b);
  if (rc) return rc;
  if (p->schedule != VD_SCHEDULE_BATCHED) return fail(VD_EINVAL, "the gradient runs the batched schedule only");
  if (!(p->gap > 0.0) || !(p->ext > 0.0)) return fail(VD_EINVAL, "the gradient needs gap > 0 and ext > 0");
  if (checkpoint != VD_CHECKPOINT_SQRT && checkpoint != VD_CHECKPOINT_ALL) return fail(VD_EINVAL, "unknown checkpoint mode");
  const int64_t n_out = batch_outputs(b);
  if (n_out > 0 && (!out_ln || !out_jac)) return fail(VD_EINVAL, "out_ln or out_jac is NULL");
  for (int64_t r = 0; r < b->n_reads; ++r)
    if (b->read_off[r + 1] - b->read_off[r] + (p->anchored ? 1 : 0) > kStripRows)
      return fail(VD_EINVAL, "the gradient supports reads of at most 256 bases (255 anchored)");
  std::lock_guard<std::mutex> lk(e->mu);
  DeviceGuard guard(e->device);
  vd_grad_stats s{};
  s.pairs = n_out;
  if ((rc = ensure_tables(e, p))) return rc;
  const bool offsets = p->quality_offsets != nullptr;
  const bool store_all = checkpoint == VD_CHECKPOINT_ALL;
  const bool f64_only = p->precision == VD_PRECISION_FLOAT64;

  // every input on the device once; reads carry the code of the forward tiers
  HostChunk c;
  c.ra = 0; c.rb = b->n_reads; c.ha = 0; c.hb = b->n_haps;
  finish_chunk_common(c, b, e->htab, offsets, p->anchored != 0);
  std::vector<RescueEntry> items;
  items.reserve((size_t)n_out);
  std::vector<int64_t> empty_slots;
  auto add = [&](int64_t r, int64_t h, int64_t o) {
    const int64_t n = b->read_off[r + 1] - b->read_off[r], m = b->hap_off[h + 1] - b->hap_off[h];
    if (n <= 0 || m <= 0) { empty_slots.push_back(o); return; }
    items.push_back(RescueEntry{(int32_t)r, (int32_t)h, o});
    s.dp_cells += n * m;
  };
  if (b->pair_read) {
    for (int64_t q = 0; q < b->n_pairs; ++q) add(b->pair_read[q], b->pair_hap[q], q);
  } else {
    int64_t o = 0;
    for (int64_t g = 0; g < b->n_regions; ++g)
      for (int64_t r = b->region_read_off[g]; r < b->region_read_off[g + 1]; ++r)
        for (int64_t h = b->region_hap_off[g]; h < b->region_hap_off[g + 1]; ++h) add(r, h, o++);
  }
  // group by kernel variant, longest haplotype first inside a group
  auto hlen = [&](const RescueEntry& x) { return b->hap_off[x.hap + 1] - b->hap_off[x.hap]; };
  std::stable_sort(items.begin(), items.end(), [&](const RescueEntry& x, const RescueEntry& y) {
    const int cx = c.read_code[x.read] & 0x1ff, cy = c.read_code[y.read] & 0x1ff;
    if (cx != cy) return cx > cy;
    return hlen(x) > hlen(y);
  });
  long long slot_bytes = 256;
  for (const RescueEntry& x : items)
    slot_bytes = std::max(slot_bytes, grad_slot_bytes(code_R(c.read_code[x.read]), (int)hlen(x), store_all));
  slot_bytes = (long long)align_up((size_t)slot_bytes, 256);
  const int grid32 = e->grid_grad[0], grid64 = e->grid_grad[1];
  const int64_t slots = (int64_t)std::max(grid32, grid64) * kWarpsPerBlock;

  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + std::max<size_t>(bytes, 1), 256); return o; };
  const int64_t read_bytes = c.read_off.back(), hap_bytes = c.hap_off.back();
  const size_t o_rb = take(read_bytes), o_rq = take(read_bytes), o_roff = take(c.read_off.size() * 8),
               o_rcode = take(c.read_code.size() * 4), o_hb = take(hap_bytes), o_hoff = take(c.hap_off.size() * 8),
               o_items = take(items.size() * sizeof(RescueEntry)), o_spill = take(items.size() * sizeof(RescueEntry)),
               o_ln = take((size_t)n_out * 8), o_jac = take((size_t)n_out * 48), o_cnt = take(8 * 8),
               o_gt = take(sizeof(GradTables)), o_scratch = take((size_t)(slots * slot_bytes));
  if ((rc = e->grad_arena.reserve(off))) return rc;
  char* d = (char*)e->grad_arena.p;
  s.scratch_bytes = (int64_t)(slots * slot_bytes);
  GradTables gt;
  GradScalars gs;
  build_grad_tables(p->gap, p->ext, p->quality_offsets, &gt, &gs);
  cudaStream_t st_ = e->stream;
  auto put = [&](size_t o, const void* src, size_t n) -> int {
    if (n) VD_CUDA(cudaMemcpyAsync(d + o, src, n, cudaMemcpyHostToDevice, st_));
    return VD_OK;
  };
  if ((rc = put(o_rb, b->read_bases + b->read_off[0], read_bytes)) || (rc = put(o_rq, b->read_quals + b->read_off[0], read_bytes)) ||
      (rc = put(o_roff, c.read_off.data(), c.read_off.size() * 8)) || (rc = put(o_rcode, c.read_code.data(), c.read_code.size() * 4)) ||
      (rc = put(o_hb, b->hap_bases + b->hap_off[0], hap_bytes)) || (rc = put(o_hoff, c.hap_off.data(), c.hap_off.size() * 8)) ||
      (rc = put(o_items, items.data(), items.size() * sizeof(RescueEntry))) || (rc = put(o_gt, &gt, sizeof(GradTables))))
    return rc;
  VD_CUDA(cudaMemsetAsync(d + o_cnt, 0, 64, st_));
  BatchView bv{};
  bv.read_bases = (const uint8_t*)(d + o_rb);
  bv.read_quals = (const uint8_t*)(d + o_rq);
  bv.read_off = (const int64_t*)(d + o_roff);
  bv.read_code = (const int32_t*)(d + o_rcode);
  bv.hap_bases = (const uint8_t*)(d + o_hb);
  bv.hap_off = (const int64_t*)(d + o_hoff);
  unsigned long long* cnt = (unsigned long long*)(d + o_cnt);
  GradView gv{};
  gv.out_ln = (double*)(d + o_ln);
  gv.out_jac = (double*)(d + o_jac);
  gv.scratch = d + o_scratch;
  gv.slot_bytes = slot_bytes;
  gv.store_all = store_all ? 1 : 0;
  gv.anchored = p->anchored ? 1 : 0;
  gv.error_flag = (int*)(cnt + 4);
  const TableSet* dt = (const TableSet*)e->dtab.p;
  const TableSet* ht = e->htab;
  VD_CUDA(cudaEventRecord(e->ev_begin, st_));
  cudaGetLastError();
  if (!items.empty()) {
    cudaError_t err;
    if (!f64_only) {
      gv.items = (const RescueEntry*)(d + o_items);
      gv.count = nullptr;
      gv.n_items = (long long)items.size();
      gv.head = cnt + 0;
      gv.spill = (RescueEntry*)(d + o_spill);
      gv.spill_count = cnt + 2;
      gv.spill_cap = (long long)items.size();
      err = launch_grad_f32(bv, gv, &dt->f32, ht->s32, (const GradTables*)(d + o_gt), gs, grid32, st_);
      if (err != cudaSuccess) return cuda_fail(err, "gradient FP32 pass launch");
      ++s.kernel_launches;
    }
    gv.items = (const RescueEntry*)(d + (f64_only ? o_items : o_spill));
    gv.count = f64_only ? nullptr : cnt + 2;
    gv.n_items = (long long)items.size();
    gv.head = cnt + 1;
    gv.spill = nullptr;
    gv.spill_count = nullptr;
    gv.spill_cap = 0;
    err = launch_grad_f64(bv, gv, &dt->f64, ht->s64, (const GradTables*)(d + o_gt), gs, grid64, st_);
    if (err != cudaSuccess) return cuda_fail(err, "gradient FP64 pass launch");
    ++s.kernel_launches;
  }
  VD_CUDA(cudaEventRecord(e->ev_end, st_));
  // outputs: the kernels write every non-empty slot; empty pairs are -inf with a zero gradient
  std::vector<double> ln((size_t)n_out), jac((size_t)n_out * 6);
  unsigned long long hc[8];
  if (n_out) {
    VD_CUDA(cudaMemcpyAsync(ln.data(), d + o_ln, (size_t)n_out * 8, cudaMemcpyDeviceToHost, st_));
    VD_CUDA(cudaMemcpyAsync(jac.data(), d + o_jac, (size_t)n_out * 48, cudaMemcpyDeviceToHost, st_));
  }
  VD_CUDA(cudaMemcpyAsync(hc, d + o_cnt, 64, cudaMemcpyDeviceToHost, st_));
  VD_CUDA(cudaStreamSynchronize(st_));
  float ms = 0.f;
  VD_CUDA(cudaEventElapsedTime(&ms, e->ev_begin, e->ev_end));
  s.kernel_ms = ms;
  const unsigned flags = (unsigned)(hc[4] & 0xffffffffu);
  if (flags & 1u) return fail(VD_EOVERFLOW, "gradient spill list overflow");
  s.fp64_pairs = f64_only ? (int64_t)items.size() : (int64_t)hc[2];
  for (int64_t o : empty_slots) {
    ln[(size_t)o] = -HUGE_VAL;
    for (int k = 0; k < 6; ++k) jac[(size_t)o * 6 + k] = 0.0;
  }
  for (int64_t k = 0; k < n_out; ++k) if (std::isnan(ln[(size_t)k])) ++s.failed_pairs;
  std::memcpy(out_ln, ln.data(), (size_t)n_out * 8);
  std::memcpy(out_jac, jac.data(), (size_t)n_out * 48);
  s.total_ms = now_ms() - t0;
  if (st) *st = s;
  return VD_OK;
}

// ---- region post-processing ------------------------------------------------------------

int vd_region_genotypes(vd_engine* e, const vd_batch* b, const vd_params* p, const unsigned char* mapping_quality,
                        const vd_genotype_options* opt, double* out_ln, double* out_values, double* out_certainty,
                        double* out_gl, int* out_guarded, vd_stats* st) {
  const double t0 = now_ms();
  if (!e) return fail(VD_EINVAL, "engine is NULL");
  int rc = validate_params(p);
  if (!rc) rc = validate_batch(b);
  if (rc) return rc;
  if (b->pair_read) return fail(VD_EINVAL, "genotypes need the region form of the batch");
  if (!opt) return fail(VD_EINVAL, "options is NULL");
  const double artifact_prior = opt->artifact_prior;
  if (!(artifact_prior < 1.0) || std::isnan(artifact_prior)) return fail(VD_EINVAL, "artifact_prior must be < 1");
  if (opt->near_tie_guard != 0 && opt->near_tie_guard != 1) return fail(VD_EINVAL, "near_tie_guard must be 0 or 1");
  for (int i = 0; i < 3; ++i) if (opt->reserved[i]) return fail(VD_EINVAL, "reserved fields must be zero");
  const int64_t G = b->n_regions;
  // host layout: rows of the regions' reads, and per-region offsets
  std::vector<int64_t> row_off, r_out(G), r_reads(G), gl_off(G + 1, 0), acc_off(G + 1, 0);
  std::vector<int32_t> row_h, r_h(G);
  std::vector<double> mq_err;
  std::vector<int64_t> row_read;
  int64_t out = 0;
  for (int64_t g = 0; g < G; ++g) {
    const int64_t r0 = b->region_read_off[g], r1 = b->region_read_off[g + 1];
    const int64_t H = b->region_hap_off[g + 1] - b->region_hap_off[g];
    if (H > 4096) return fail(VD_EINVAL, "genotypes support at most 4096 haplotypes per region");
    r_out[g] = out;
    r_reads[g] = r1 - r0;
    r_h[g] = (int32_t)H;
    const int64_t P = H * (H + 1) / 2;
    const int64_t M = artifact_prior < 0.0 ? 1 : 7 + (artifact_prior > 0.0 ? 4 * H : 0);
    gl_off[g + 1] = gl_off[g] + P;
    acc_off[g + 1] = acc_off[g] + P * M;
    for (int64_t r = r0; r < r1; ++r) {
      row_off.push_back(out + (r - r0) * H);
      row_h.push_back((int32_t)H);
      row_read.push_back(r);
      // caller/native/caller/molecule_rows.py:4 _MQ_ERROR
      const unsigned q = mapping_quality ? mapping_quality[r] : 60u;
      mq_err.push_back(std::pow(10.0, -(double)std::min(q, 60u) / 10.0));
    }
    out += (r1 - r0) * H;
  }
  const int64_t n_rows = (int64_t)row_off.size(), n_out = out;
  if (gl_off[G] > 0 && !out_gl) return fail(VD_EINVAL, "out_gl is NULL");
  const bool guard = opt->near_tie_guard == 1 && p->precision != VD_PRECISION_FLOAT64;
  std::vector<int> flags((size_t)G, 0);
  vd_plan* pl = nullptr;
  if ((rc = vd_plan_create(e, b, p, &pl))) return rc;
  vd_stats s{};
  if ((rc = vd_plan_run(pl, &s))) { vd_plan_destroy(pl); return rc; }
  {
    std::lock_guard<std::mutex> lk(e->mu);
    DeviceGuard dguard(e->device);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + std::max<size_t>(bytes, 1), 256); return o; };
    const size_t o_roff = take(n_rows * 8), o_rh = take(n_rows * 4), o_mq = take(n_rows * 8),
                 o_gout = take(G * 8), o_greads = take(G * 8), o_gh = take(G * 4), o_gloff = take((G + 1) * 8),
                 o_accoff = take((G + 1) * 8), o_val = take(n_out * 8), o_cert = take(n_rows * 8),
                 o_gl = take(gl_off[G] * 8), o_acc = take(acc_off[G] * 8), o_flag = take(G * 4);
    rc = e->geno_arena.reserve(off);
    char* d = (char*)e->geno_arena.p;
    cudaStream_t sm = e->stream;
    auto put = [&](size_t o, const void* src, size_t n) -> int {
      if (n) VD_CUDA(cudaMemcpyAsync(d + o, src, n, cudaMemcpyHostToDevice, sm));
      return VD_OK;
    };
    if (!rc && !(rc = put(o_roff, row_off.data(), n_rows * 8)) && !(rc = put(o_rh, row_h.data(), n_rows * 4)) &&
        !(rc = put(o_mq, mq_err.data(), n_rows * 8)) && !(rc = put(o_gout, r_out.data(), G * 8)) &&
        !(rc = put(o_greads, r_reads.data(), G * 8)) && !(rc = put(o_gh, r_h.data(), G * 4)) &&
        !(rc = put(o_gloff, gl_off.data(), (G + 1) * 8)) && !(rc = put(o_accoff, acc_off.data(), (G + 1) * 8))) {
      const double* dln = (const double*)(pl->base + pl->L.o_out);
      cudaError_t err = cudaEventRecord(e->ev_begin, sm);
      if (err == cudaSuccess)
        err = launch_genotype_rows(dln, (const int64_t*)(d + o_roff), (const int32_t*)(d + o_rh),
                                   (const double*)(d + o_mq), n_rows, (double*)(d + o_val), (double*)(d + o_cert),
                                   e->sm_count, sm);
      if (err == cudaSuccess)
        err = launch_genotype_gl((const double*)(d + o_val), (const int64_t*)(d + o_gout),
                                 (const int64_t*)(d + o_greads), (const int32_t*)(d + o_gh),
                                 (const int64_t*)(d + o_gloff), (const int64_t*)(d + o_accoff), G, artifact_prior,
                                 (double*)(d + o_acc), (double*)(d + o_gl), e->sm_count, sm);
      if (err == cudaSuccess && guard)
        err = launch_genotype_ties((const double*)(d + o_gl), (const int64_t*)(d + o_gloff),
                                   (const int32_t*)(d + o_gh), (const int64_t*)(d + o_greads), G, (int*)(d + o_flag),
                                   sm);
      if (err == cudaSuccess) err = cudaEventRecord(e->ev_end, sm);
      std::vector<double> cert((size_t)n_rows);
      if (err == cudaSuccess && gl_off[G])
        err = cudaMemcpyAsync(out_gl, d + o_gl, gl_off[G] * 8, cudaMemcpyDeviceToHost, sm);
      if (err == cudaSuccess && out_values && n_out)
        err = cudaMemcpyAsync(out_values, d + o_val, n_out * 8, cudaMemcpyDeviceToHost, sm);
      if (err == cudaSuccess && out_certainty && n_rows)
        err = cudaMemcpyAsync(cert.data(), d + o_cert, n_rows * 8, cudaMemcpyDeviceToHost, sm);
      if (err == cudaSuccess && out_ln && n_out)
        err = cudaMemcpyAsync(out_ln, dln, n_out * 8, cudaMemcpyDeviceToHost, sm);
      if (err == cudaSuccess && guard && G)
        err = cudaMemcpyAsync(flags.data(), d + o_flag, G * 4, cudaMemcpyDeviceToHost, sm);
      if (err == cudaSuccess) err = cudaStreamSynchronize(sm);
      float ms = 0.f;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e->ev_begin, e->ev_end);
      if (err != cudaSuccess) {
        rc = cuda_fail(err, "genotype post-processing");
      } else {
        if (out_certainty)
          for (int64_t k = 0; k < n_rows; ++k) out_certainty[row_read[k]] = cert[(size_t)k];
        s.kernel_ms += ms;
        s.kernel_launches += guard ? 3 : 2;
        s.d2h_bytes = gl_off[G] * 8 + (out_values ? n_out * 8 : 0) + (out_certainty ? n_rows * 8 : 0) +
                      (out_ln ? n_out * 8 : 0) + (guard ? G * 4 : 0);
      }
    }
  }
  vd_plan_destroy(pl);
  if (rc) return rc;
  if (out_guarded) for (int64_t g = 0; g < G; ++g) out_guarded[g] = flags[(size_t)g];

  // near ties: the flagged regions again, in FP64, their results in place
  std::vector<int64_t> tied;
  for (int64_t g = 0; g < G; ++g) if (flags[(size_t)g]) tied.push_back(g);
  if (!tied.empty()) {
    std::vector<unsigned char> rb, rq, hb, mq;
    std::vector<int64_t> ro{0}, ho{0}, rro{0}, rho{0};
    for (int64_t g : tied) {
      const int64_t r0 = b->region_read_off[g], r1 = b->region_read_off[g + 1];
      const int64_t h0 = b->region_hap_off[g], h1 = b->region_hap_off[g + 1];
      for (int64_t r = r0; r < r1; ++r) {
        const int64_t a0 = b->read_off[r], a1 = b->read_off[r + 1];
        rb.insert(rb.end(), b->read_bases + a0, b->read_bases + a1);
        rq.insert(rq.end(), b->read_quals + a0, b->read_quals + a1);
        ro.push_back(ro.back() + (a1 - a0));
        mq.push_back(mapping_quality ? mapping_quality[r] : (unsigned char)60);
      }
      for (int64_t h = h0; h < h1; ++h) {
        const int64_t c0 = b->hap_off[h], c1 = b->hap_off[h + 1];
        hb.insert(hb.end(), b->hap_bases + c0, b->hap_bases + c1);
        ho.push_back(ho.back() + (c1 - c0));
      }
      rro.push_back(rro.back() + (r1 - r0));
      rho.push_back(rho.back() + (h1 - h0));
    }
    vd_batch sub{};
    sub.read_bases = rb.data();
    sub.read_quals = rq.data();
    sub.read_off = ro.data();
    sub.n_reads = (int64_t)ro.size() - 1;
    sub.hap_bases = hb.data();
    sub.hap_off = ho.data();
    sub.n_haps = (int64_t)ho.size() - 1;
    sub.region_read_off = rro.data();
    sub.region_hap_off = rho.data();
    sub.n_regions = (int64_t)tied.size();
    vd_params p64 = *p;
    p64.precision = VD_PRECISION_FLOAT64;
    vd_genotype_options o64 = *opt;
    o64.near_tie_guard = 0;
    int64_t sub_out = 0, sub_gl = 0;
    for (size_t k = 0; k < tied.size(); ++k) {
      const int64_t g = tied[k], H = r_h[(size_t)g];
      sub_out += r_reads[(size_t)g] * H;
      sub_gl += H * (H + 1) / 2;
    }
    std::vector<double> ln2((size_t)sub_out), val2((size_t)sub_out), cert2((size_t)sub.n_reads), gl2((size_t)sub_gl);
    vd_stats s2{};
    rc = vd_region_genotypes(e, &sub, &p64, mq.data(), &o64, ln2.data(), val2.data(), cert2.data(), gl2.data(),
                             nullptr, &s2);
    if (rc) return rc;
    int64_t so = 0, sg = 0, sr = 0;
    for (int64_t g : tied) {
      const int64_t H = r_h[(size_t)g], nr = r_reads[(size_t)g], P = H * (H + 1) / 2;
      for (int64_t k = 0; k < nr * H; ++k) {
        if (out_ln) out_ln[r_out[(size_t)g] + k] = ln2[(size_t)(so + k)];
        if (out_values) out_values[r_out[(size_t)g] + k] = val2[(size_t)(so + k)];
      }
      for (int64_t k = 0; k < P; ++k) out_gl[gl_off[(size_t)g] + k] = gl2[(size_t)(sg + k)];
      if (out_certainty)
        for (int64_t k = 0; k < nr; ++k) out_certainty[b->region_read_off[g] + k] = cert2[(size_t)(sr + k)];
      so += nr * H;
      sg += P;
      sr += nr;
    }
    s.kernel_ms += s2.kernel_ms;
    s.kernel_launches += s2.kernel_launches;
    s.rescued_fp64 += s2.pairs;
  }
  s.total_ms = now_ms() - t0;
  if (st) *st = s;
  return VD_OK;
}

// ---- reference-shaped entry points --------------------------------------------------

namespace {

// Pack pointer-array inputs (the reference's ctypes calling convention) into a
// vd_batch of explicit pairs; identical (pointer, length) reads and
// haplotypes are stored once.
struct PackedPairs {
  std::vector<unsigned char> rb, rq, hb;
  std::vector<int64_t> roff{0}, hoff{0};
  std::vector<int32_t> pr, ph;
  vd_batch batch{};
};

struct PtrKey {
  const void* a;
  const void* b;
  int n;
  bool operator==(const PtrKey& o) const { return a == o.a && b == o.b && n == o.n; }
};
struct PtrHash {
  size_t operator()(const PtrKey& k) const {
    return std::hash<const void*>()(k.a) * 31 + std::hash<const void*>()(k.b) * 7 + (size_t)k.n;
  }
};

void pack_pairs(const char* const* reads, const unsigned char* const* quals, const int* rn,
                const char* const* haps, const int* hn, int count, PackedPairs& pp) {
  std::unordered_map<PtrKey, int32_t, PtrHash> rid, hid;
  pp.pr.resize(count);
  pp.ph.resize(count);
  for (int p = 0; p < count; ++p) {
    const int n = std::max(0, rn[p]);
    PtrKey rk{reads[p], quals[p], n};
    auto it = rid.find(rk);
    if (it == rid.end()) {
      const int32_t id = (int32_t)pp.roff.size() - 1;
      pp.rb.insert(pp.rb.end(), (const unsigned char*)reads[p], (const unsigned char*)reads[p] + n);
      pp.rq.insert(pp.rq.end(), quals[p], quals[p] + n);
      pp.roff.push_back((int64_t)pp.rb.size());
      it = rid.emplace(rk, id).first;
    }
    pp.pr[p] = it->second;
    const int m = std::max(0, hn[p]);
    PtrKey hk{haps[p], nullptr, m};
    auto jt = hid.find(hk);
    if (jt == hid.end()) {
      const int32_t id = (int32_t)pp.hoff.size() - 1;
      pp.hb.insert(pp.hb.end(), (const unsigned char*)haps[p], (const unsigned char*)haps[p] + m);
      pp.hoff.push_back((int64_t)pp.hb.size());
      jt = hid.emplace(hk, id).first;
    }
    pp.ph[p] = jt->second;
  }
  vd_batch& b = pp.batch;
  b.read_bases = pp.rb.data();
  b.read_quals = pp.rq.data();
  b.read_off = pp.roff.data();
  b.n_reads = (int64_t)pp.roff.size() - 1;
  b.hap_bases = pp.hb.data();
  b.hap_off = pp.hoff.data();
  b.n_haps = (int64_t)pp.hoff.size() - 1;
  b.pair_read = pp.pr.data();
  b.pair_hap = pp.ph.data();
  b.n_pairs = count;
}

vd_params fixed_params(int mode) {
  vd_params p{};
  p.gap = 0.001;
  p.ext = 0.1;
  p.anchored = mode == 1 ? 1 : 0;
  p.precision = default_precision();
  return p;
}

double single_pair(const char* read, const unsigned char* qual, int n, const char* hap, int m, double gap,
                   double ext, int anchored) {
  if (n <= 0 || m <= 0) return -HUGE_VAL;
  vd_engine* e = nullptr;
  if (default_engine(&e)) return NAN;
  int64_t roff[2] = {0, n}, hoff[2] = {0, m}, rr[2] = {0, 1}, hr[2] = {0, 1};
  vd_batch b{};
  b.read_bases = (const unsigned char*)read;
  b.read_quals = qual;
  b.read_off = roff;
  b.n_reads = 1;
  b.hap_bases = (const unsigned char*)hap;
  b.hap_off = hoff;
  b.n_haps = 1;
  b.region_read_off = rr;
  b.region_hap_off = hr;
  b.n_regions = 1;
  vd_params p{};
  p.gap = gap;
  p.ext = ext;
  p.anchored = anchored;
  p.precision = default_precision();
  double out = NAN;
  if (vd_forward(e, &b, &p, &out, nullptr)) return NAN;
  return out;
}

}  // namespace

int vd_pairhmm_pairs(const char* const* reads, const unsigned char* const* quals, const int* rn,
                     const char* const* haps, const int* hn, int count, int mode, int lanes, double* out) {
  (void)lanes;
  if (count < 0 || mode < 0 || mode > 2) return fail(VD_EINVAL, "count < 0 or mode outside 0..2");
  if (count == 0) return VD_OK;
  if (!reads || !quals || !rn || !haps || !hn || !out) return fail(VD_EINVAL, "NULL argument");
  vd_engine* e = nullptr;
  int rc = default_engine(&e);
  if (rc) return rc;
  PackedPairs pp;
  pack_pairs(reads, quals, rn, haps, hn, count, pp);
  vd_params p = fixed_params(mode);
  return vd_forward(e, &pp.batch, &p, out, nullptr);
}

int vd_trie_many(const char* const* reads, const unsigned char* const* quals, const int* rn, int nr,
                 const char* const* haps, const int* hn, int nh, int mode, int lanes, double* out,
                 uint64_t* cells) {
  (void)lanes;
  if (nr < 0 || nh < 0 || mode < 0 || mode > 2) return fail(VD_EINVAL, "nr/nh < 0 or mode outside 0..2");
  if (cells) *cells = 0;
  if (nr == 0 || nh == 0) return VD_OK;
  if (!reads || !quals || !rn || !haps || !hn || !out) return fail(VD_EINVAL, "NULL argument");
  vd_engine* e = nullptr;
  int rc = default_engine(&e);
  if (rc) return rc;
  std::vector<unsigned char> rb, rq, hb;
  std::vector<int64_t> roff{0}, hoff{0};
  for (int r = 0; r < nr; ++r) {
    const int n = std::max(0, rn[r]);
    rb.insert(rb.end(), (const unsigned char*)reads[r], (const unsigned char*)reads[r] + n);
    rq.insert(rq.end(), quals[r], quals[r] + n);
    roff.push_back((int64_t)rb.size());
  }
  for (int h = 0; h < nh; ++h) {
    const int m = std::max(0, hn[h]);
    hb.insert(hb.end(), (const unsigned char*)haps[h], (const unsigned char*)haps[h] + m);
    hoff.push_back((int64_t)hb.size());
  }
  int64_t rr[2] = {0, nr}, hr[2] = {0, nh};
  vd_batch b{};
  b.read_bases = rb.data();
  b.read_quals = rq.data();
  b.read_off = roff.data();
  b.n_reads = nr;
  b.hap_bases = hb.data();
  b.hap_off = hoff.data();
  b.n_haps = nh;
  b.region_read_off = rr;
  b.region_hap_off = hr;
  b.n_regions = 1;
  vd_params p = fixed_params(mode);
  vd_stats s{};
  rc = vd_forward(e, &b, &p, out, &s);
  if (!rc && cells) *cells = (uint64_t)s.dp_cells;
  return rc;
}

int vd_read_haplotype_batch_mode(const char* read, const unsigned char* qual, int n, const char* const* haps,
                                 const int* lengths, int count, double gap, double ext, double* out, int mode) {
  (void)mode;
  if (count < 0) return fail(VD_EINVAL, "count < 0");
  if (count == 0) return VD_OK;
  if (!haps || !lengths || !out || (n > 0 && (!read || !qual))) return fail(VD_EINVAL, "NULL argument");
  vd_engine* e = nullptr;
  int rc = default_engine(&e);
  if (rc) return rc;
  std::vector<unsigned char> hb;
  std::vector<int64_t> hoff{0};
  for (int h = 0; h < count; ++h) {
    const int m = std::max(0, lengths[h]);
    hb.insert(hb.end(), (const unsigned char*)haps[h], (const unsigned char*)haps[h] + m);
    hoff.push_back((int64_t)hb.size());
  }
  int64_t roff[2] = {0, std::max(0, n)}, rr[2] = {0, 1}, hr[2] = {0, count};
  vd_batch b{};
  b.read_bases = (const unsigned char*)read;
  b.read_quals = qual;
  b.read_off = roff;
  b.n_reads = 1;
  b.hap_bases = hb.data();
  b.hap_off = hoff.data();
  b.n_haps = count;
  b.region_read_off = rr;
  b.region_hap_off = hr;
  b.n_regions = 1;
  vd_params p{};
  p.gap = gap;
  p.ext = ext;
  p.precision = default_precision();
  return vd_forward(e, &b, &p, out, nullptr);
}

double vd_read_haplotype(const char* read, const unsigned char* qual, int n, const char* hap, int m, double gap,
                         double ext) {
  return single_pair(read, qual, n, hap, m, gap, ext, 0);
}

double vd_anchored_pairhmm(const char* read, const unsigned char* qual, int n, const char* hap, int m, double gap,
                           double ext) {
  return single_pair(read, qual, n, hap, m, gap, ext, 1);
}

}  // extern "C"
