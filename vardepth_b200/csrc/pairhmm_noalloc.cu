// An entry point that allocates nothing: vd_forward_region_noalloc.
//
// Some callers cannot call cudaMalloc: code that runs while another component
// owns all device allocation (a framework's caching allocator or a fixed
// memory pool that must not be bypassed), code in processes that forbid
// driver allocations after start-up, and code that must never block on the
// allocator.  For them this entry point scores one region (every read against
// every haplotype) whose inputs and outputs the caller already holds in device
// memory, and keeps all of its scratch -- tier counters, the work codes and
// haplotype lists it builds on the device, the rescue lists and the strip
// boundaries of the robust tier, and the model tables -- in one file-scope
// static __device__ array of kNoAllocBytes.  Every GPU that loads this library
// holds that array until the process exits.
//
// In host code the array's name is only a host-side stand-in; its device
// address is taken once per device, with that device current, by
// cudaGetSymbolAddress during the first call on the device, and passed to the
// kernels from then on.  That first call should come before any stream capture.
// Every call reuses the same array and finds the previous call's contents in
// it: the counters that must start at zero are cleared at the start of each
// call, the lists are read only up to those counters.  Overlapping calls on
// one device would race on its array; calls from several host threads on the
// same device are serialised by a per-device lock (calls on different devices
// use different arrays and run side by side).  The caller's buffers are
// checked to be device memory of the chosen device before anything is
// enqueued, and a call that fails after enqueueing work waits for it before
// returning.
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/vardepth_pairhmm.h"
#include "pairhmm_kernel.cuh"
#include "pairhmm_launch.h"

namespace vd {
namespace {

// Limits of one call (checked before anything runs; lengths are checked on
// the device, since the offsets live there).
constexpr int64_t kNaMaxPairs = 131072;   // reads x haplotypes
constexpr int64_t kNaMaxReads = 131072;
constexpr int64_t kNaMaxHaps = 4096;
constexpr int kNaMaxReadLen = 255;         // plus the anchored emulator row: one 256-row strip
constexpr int kNaMaxHapLen = 1023;
constexpr int kNaRobustBlocks = 32;        // grid of the robust tier (its strip scratch is per warp)
constexpr int kNaRobustWarps = kNaRobustBlocks * kWarpsPerBlock;

constexpr size_t na_align(size_t v) { return (v + 255) / 256 * 256; }

// Layout of the static scratch (byte offsets).
constexpr size_t kOffCnt = 0;  // 16 x u64: [0..2] work heads, [3],[4] spill counts, [5] overflow,
                               // [8] length error, [9] non-empty haplotypes
constexpr size_t kOffTab32 = 256;
constexpr size_t kOffTab64 = na_align(kOffTab32 + sizeof(Tables<float>));
constexpr size_t kOffCode = na_align(kOffTab64 + sizeof(Tables<double>));
constexpr size_t kOffHapSel = na_align(kOffCode + sizeof(int32_t) * kNaMaxReads);
constexpr size_t kOffOutSel = na_align(kOffHapSel + sizeof(int32_t) * kNaMaxHaps);
constexpr size_t kOffSpill1 = na_align(kOffOutSel + sizeof(int64_t) * kNaMaxPairs);
constexpr size_t kOffSpill2 = na_align(kOffSpill1 + sizeof(RescueEntry) * kNaMaxPairs);
constexpr size_t kOffStrip = na_align(kOffSpill2 + sizeof(RescueEntry) * kNaMaxPairs);
constexpr size_t kNoAllocBytes = na_align(kOffStrip + sizeof(double2) * (kNaMaxHapLen + 1) * kNaRobustWarps);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Haplotype list of the region: the non-empty haplotypes in order, and a
// length check.  One block.
__global__ void na_prep_haps(const int64_t* __restrict__ hap_off, int n_haps, unsigned char* scratch) {
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(scratch + kOffCnt);
  int32_t* hap_sel = reinterpret_cast<int32_t*>(scratch + kOffHapSel);
  __shared__ int warp_sums[32];
  __shared__ int base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int start = 0; start < n_haps; start += blockDim.x) {
    const int h = start + threadIdx.x;
    int keep = 0;
    if (h < n_haps) {
      const int64_t m = hap_off[h + 1] - hap_off[h];
      if (m > kNaMaxHapLen || m < 0) atomicCAS(&cnt[8], 0ull, 2ull);  // the first limit found is reported
      keep = m > 0 ? 1 : 0;
    }
    // block-wide exclusive scan of keep (order-preserving compaction)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = keep;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      int w = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += v;
      }
      if (lane < nw) warp_sums[lane] = w;  // inclusive warp totals
    }
    __syncthreads();
    const int before = (warp ? warp_sums[warp - 1] : 0) + incl - keep;
    if (keep) hap_sel[base + before] = h;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) base += before + keep;
    __syncthreads();
  }
  if (threadIdx.x == 0) cnt[9] = (unsigned long long)base;
}

// Per-read kernel codes, length checks, -inf for every output, and the output
// slot of every (read, non-empty haplotype).
__global__ void na_prep_reads(const unsigned char* __restrict__ read_quals, const int64_t* __restrict__ read_off,
                              int n_reads, int n_haps, int anchored, double* __restrict__ out,
                              unsigned char* scratch) {
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(scratch + kOffCnt);
  const Tables<float>* tab = reinterpret_cast<const Tables<float>*>(scratch + kOffTab32);
  int32_t* code = reinterpret_cast<int32_t*>(scratch + kOffCode);
  const int32_t* hap_sel = reinterpret_cast<const int32_t*>(scratch + kOffHapSel);
  int64_t* out_sel = reinterpret_cast<int64_t*>(scratch + kOffOutSel);
  const int nh_ne = (int)cnt[9];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t r = tid; r < n_reads; r += stride) {
    const int64_t o = read_off[r];
    const int64_t n = read_off[r + 1] - o;
    if (n > kNaMaxReadLen || n < 0) atomicCAS(&cnt[8], 0ull, 1ull);
    bool gen = false;
    for (int64_t i = 0; i < n && i < kNaMaxReadLen; ++i) gen |= tab->general[read_quals[o + i]] != 0;
    const int rows = (int)n + anchored;
    const int R = min(kMaxR, max(1, (rows + kWarp - 1) / kWarp));
    code[r] = make_code(R, gen, false);
  }
  for (int64_t k = tid; k < (int64_t)n_reads * n_haps; k += stride) out[k] = -HUGE_VAL;
  for (int64_t k = tid; k < (int64_t)n_reads * nh_ne; k += stride) {
    const int64_t r = k / nh_ne, j = k - r * nh_ne;
    out_sel[k] = r * n_haps + hap_sel[j];
  }
}

// Primary tier over the region: work item r is read r against the non-empty
// haplotypes, derived here instead of read from a host-built list.
template <typename T, bool ANCH>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp, MinBlocks<T>::value)
na_primary(const BatchView bv, const QueueView qv, const Scalars<T> sc, int n_reads, unsigned char* scratch) {
  __shared__ Tables<T> tab;
  {
    const Tables<T>* g = reinterpret_cast<const Tables<T>*>(scratch + (sizeof(T) == 4 ? kOffTab32 : kOffTab64));
    const int words = (int)(sizeof(Tables<T>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(g);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const unsigned long long* cnt = reinterpret_cast<const unsigned long long*>(scratch + kOffCnt);
  if (cnt[8] != 0) return;  // a length limit was exceeded: nothing runs
  const int nh_ne = (int)cnt[9];
  const int lane = threadIdx.x & (kWarp - 1);
  using T2 = typename Vec2<T>::type;
  T2* strip = reinterpret_cast<T2*>(qv.scratch);  // not used: one strip per read in this tier
  for (;;) {
    unsigned long long i = 0;
    if (lane == 0) i = atomicAdd(qv.head, 1ull);
    i = __shfl_sync(0xffffffffu, i, 0);
    if ((long long)i >= n_reads) break;
    const int n = (int)(bv.read_off[i + 1] - bv.read_off[i]);
    if (n <= 0 || nh_ne == 0) continue;
    ItemRef it;
    it.w.read = (int32_t)i;
    it.w.nhap = nh_ne;
    it.w.hap_begin = 0;
    it.w.out_begin = (int64_t)i * nh_ne;
    it.w.code = bv.read_code[i];
    it.w.read2 = -1;
    it.w.out2_begin = 0;
    it.use_sel = true;
    it.tier = 0;
    dispatch<T, ANCH>(it.w.code, bv, qv, it, &tab, sc, lane, strip);
  }
}

}  // namespace
}  // namespace vd

namespace vd {
namespace {

struct NaDevice {
  std::mutex mu;                     // one call at a time on this device: the calls share its scratch
  Tables<float> t32;                 // staging of the model tables (filled on the host, copied into the scratch)
  Tables<double> t64;
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch on this device
  int grid32[2] = {0, 0};            // [anchored] blocks of na_primary<float>
  int grid64[2] = {0, 0};            // [anchored] blocks of na_primary<double>
  int rescue[2] = {0, 0};            // [anchored] blocks of the FP64 rescue tier
};
constexpr int kNaMaxDevices = 64;
NaDevice g_na[kNaMaxDevices];

int na_fail(int code, const std::string& msg) { return report_error(code, msg.c_str()); }

int na_cuda(cudaError_t e, const char* what) {
  cudaGetLastError();
  return na_fail(VD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define NA_CUDA(call)                                       \
  do {                                                      \
    cudaError_t na_err_ = (call);                           \
    if (na_err_ != cudaSuccess) return na_cuda(na_err_, #call); \
  } while (0)

// A caller buffer must be device (or managed) memory of the call's device: a
// host pointer handed to the kernels would fault.  cudaPointerGetAttributes
// allocates nothing.
bool na_on_device(const void* p, int device) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

// Per-device set-up, with the device current: the scratch address and the
// grid sizes.  Runs during the first call on the device.
int na_setup(int device) {
  NaDevice& d = g_na[device];
  if (d.ready) return VD_OK;
  void* ptr = nullptr;
  NA_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
  d.scratch = static_cast<unsigned char*>(ptr);
  int sms = 0, b = 0;
  NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, na_primary<float, false>, kWarpsPerBlock * kWarp, 0));
  d.grid32[0] = std::max(1, b) * sms;
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, na_primary<float, true>, kWarpsPerBlock * kWarp, 0));
  d.grid32[1] = std::max(1, b) * sms;
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, na_primary<double, false>, kWarpsPerBlock * kWarp, 0));
  d.grid64[0] = std::max(1, b) * sms;
  NA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, na_primary<double, true>, kWarpsPerBlock * kWarp, 0));
  d.grid64[1] = std::max(1, b) * sms;
  for (int a = 0; a < 2; ++a) {
    NA_CUDA(occupancy_f64(a != 0, &b));
    d.rescue[a] = std::max(1, b) * sms;
  }
  d.ready = true;
  return VD_OK;
}

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" int vd_forward_region_noalloc(int device, const unsigned char* read_bases, const unsigned char* read_quals,
                                         const int64_t* read_off, int64_t n_reads, const unsigned char* hap_bases,
                                         const int64_t* hap_off, int64_t n_haps, const vd_params* params,
                                         double* out, void* stream) {
  // arguments and limits, on the host, before anything is enqueued
  if (!params) return na_fail(VD_EINVAL, "params is NULL");
  if (!(params->gap >= 0.0 && params->gap < 0.5) || !(params->ext >= 0.0 && params->ext < 1.0) ||
      (params->anchored != 0 && params->anchored != 1) ||
      (params->precision != VD_PRECISION_MIXED && params->precision != VD_PRECISION_FLOAT64))
    return na_fail(VD_EINVAL, "invalid params (gap in [0,0.5), ext in [0,1), anchored 0/1, known precision)");
  if (params->schedule != VD_SCHEDULE_BATCHED)
    return na_fail(VD_EINVAL, "this call runs the batched schedule only (schedule must be 0)");
  for (int i = 0; i < 3; ++i)
    if (params->reserved[i]) return na_fail(VD_EINVAL, "reserved fields must be zero");
  if (params->quality_offsets)
    for (int i = 0; i < 4; ++i)
      if (!std::isfinite(params->quality_offsets[i])) return na_fail(VD_EINVAL, "quality offsets must be finite");
  if (n_reads < 0 || n_haps < 0) return na_fail(VD_EINVAL, "negative counts");
  if (n_reads > kNaMaxReads || n_haps > kNaMaxHaps || n_reads * n_haps > kNaMaxPairs)
    return na_fail(VD_EINVAL, "vd_forward_region_noalloc: at most 131072 reads, 4096 haplotypes and 131072 "
                              "pairs per call (its scratch is a fixed 8 MiB array); split the region");
  if (n_reads == 0 || n_haps == 0) return VD_OK;
  if (!read_bases || !read_quals || !read_off || !hap_bases || !hap_off || !out)
    return na_fail(VD_EINVAL, "NULL device pointer");
  if (device < 0 || device >= kNaMaxDevices) return na_fail(VD_ENODEV, "device index out of range");

  std::lock_guard<std::mutex> lk(g_na[device].mu);
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return na_fail(VD_ENODEV, "cannot select the CUDA device");
  }
  struct Restore {
    int prev;
    ~Restore() { if (prev >= 0) cudaSetDevice(prev); }
  } restore{prev};
  int rc = na_setup(device);
  if (rc) return rc;
  NaDevice& d = g_na[device];
  {
    const void* bufs[6] = {read_bases, read_quals, read_off, hap_bases, hap_off, out};
    static const char* names[6] = {"read_bases", "read_quals", "read_off", "hap_bases", "hap_off", "out"};
    for (int i = 0; i < 6; ++i)
      if (!na_on_device(bufs[i], device))
        return na_fail(VD_EINVAL, std::string("vd_forward_region_noalloc: ") + names[i] +
                                      " is not device memory of the selected device");
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // once work is enqueued, an early return waits for it first: kernels still
  // running would otherwise share the scratch with the next call
  struct Drain {
    cudaStream_t s;
    bool armed = false;
    ~Drain() { if (armed) { cudaStreamSynchronize(s); cudaGetLastError(); } }
  } drain{s};
  unsigned char* sc = d.scratch;
  const bool anch = params->anchored != 0;
  const bool f64 = params->precision == VD_PRECISION_FLOAT64;

  // model tables into the scratch; the call waits for the stream at its end,
  // so the staging tables are not rewritten while the copy is pending
  Scalars<float> s32;
  Scalars<double> s64;
  build_model_tables(params->gap, params->ext, params->quality_offsets, &d.t32, &d.t64, &s32, &s64);
  drain.armed = true;
  NA_CUDA(cudaMemcpyAsync(sc + kOffTab32, &d.t32, sizeof(d.t32), cudaMemcpyHostToDevice, s));
  NA_CUDA(cudaMemcpyAsync(sc + kOffTab64, &d.t64, sizeof(d.t64), cudaMemcpyHostToDevice, s));
  // the previous call's counters and lists are still in the array: the
  // counters are cleared here; the lists are only read up to their counts
  NA_CUDA(cudaMemsetAsync(sc + kOffCnt, 0, 16 * sizeof(unsigned long long), s));
  na_prep_haps<<<1, 256, 0, s>>>(hap_off, (int)n_haps, sc);
  NA_CUDA(cudaGetLastError());
  na_prep_reads<<<(int)std::min<int64_t>(1024, (n_reads * n_haps + 255) / 256 + 1), 256, 0, s>>>(
      read_quals, read_off, (int)n_reads, (int)n_haps, anch ? 1 : 0, out, sc);
  NA_CUDA(cudaGetLastError());

  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(sc + kOffCnt);
  BatchView bv{};
  bv.read_bases = read_bases;
  bv.read_quals = read_quals;
  bv.read_off = read_off;
  bv.read_code = reinterpret_cast<const int32_t*>(sc + kOffCode);
  bv.hap_bases = hap_bases;
  bv.hap_off = hap_off;
  bv.hap_sel = reinterpret_cast<const int32_t*>(sc + kOffHapSel);
  bv.out_sel = reinterpret_cast<const int64_t*>(sc + kOffOutSel);
  bv.out = out;
  QueueView q{};
  q.items = nullptr;
  q.head = cnt + 0;
  q.spill = reinterpret_cast<RescueEntry*>(sc + kOffSpill1);
  q.spill_count = cnt + 3;
  q.spill_cap = kNaMaxPairs;
  q.scratch = sc + kOffStrip;
  q.scratch_stride = kNaMaxHapLen + 1;
  q.error_flag = reinterpret_cast<int*>(cnt + 5);
  // primary tier: FP32 (or FP64 when asked), work items derived on the device
  if (f64) {
    if (anch) na_primary<double, true><<<d.grid64[1], kWarpsPerBlock * kWarp, 0, s>>>(bv, q, s64, (int)n_reads, sc);
    else na_primary<double, false><<<d.grid64[0], kWarpsPerBlock * kWarp, 0, s>>>(bv, q, s64, (int)n_reads, sc);
  } else {
    if (anch) na_primary<float, true><<<d.grid32[1], kWarpsPerBlock * kWarp, 0, s>>>(bv, q, s32, (int)n_reads, sc);
    else na_primary<float, false><<<d.grid32[0], kWarpsPerBlock * kWarp, 0, s>>>(bv, q, s32, (int)n_reads, sc);
  }
  NA_CUDA(cudaGetLastError());
  // rescue tiers on the spill lists, with the library's own kernels
  const Tables<double>* t64 = reinterpret_cast<const Tables<double>*>(sc + kOffTab64);
  BatchView rv = bv;
  rv.hap_sel = nullptr;
  rv.out_sel = nullptr;
  if (!f64) {
    QueueView q1 = q;
    q1.entries = reinterpret_cast<const RescueEntry*>(sc + kOffSpill1);
    q1.count = cnt + 3;
    q1.n_items = kNaMaxPairs;
    q1.head = cnt + 1;
    q1.spill = reinterpret_cast<RescueEntry*>(sc + kOffSpill2);
    q1.spill_count = cnt + 4;
    NA_CUDA(launch_f64(anch, rv, q1, t64, s64, 1, d.rescue[anch], s));
  }
  QueueView q2 = q;
  q2.entries = reinterpret_cast<const RescueEntry*>(sc + (f64 ? kOffSpill1 : kOffSpill2));
  q2.count = cnt + (f64 ? 3 : 4);
  q2.n_items = kNaMaxPairs;
  q2.head = cnt + 2;
  q2.spill = nullptr;
  q2.spill_count = nullptr;
  q2.spill_cap = 0;
  NA_CUDA(launch_f64(anch, rv, q2, t64, s64, 2, std::min(d.rescue[anch], kNaRobustBlocks), s));
  // length checks and the overflow flag come back with the stream
  unsigned long long h[16];
  NA_CUDA(cudaMemcpyAsync(h, sc + kOffCnt, sizeof(h), cudaMemcpyDeviceToHost, s));
  NA_CUDA(cudaStreamSynchronize(s));
  drain.armed = false;
  if (h[8] == 1) return na_fail(VD_EINVAL, "vd_forward_region_noalloc: reads are limited to 255 bases");
  if (h[8] == 2) return na_fail(VD_EINVAL, "vd_forward_region_noalloc: haplotypes are limited to 1023 bases");
  if (h[5]) return na_fail(VD_EOVERFLOW, "rescue list overflow");
  return VD_OK;
}
