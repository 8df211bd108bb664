// The pair-list drop-in: vd_score_pair_list and its host-only plan.
//
// The reference's Python entry (caller/native/caller/accelerator.py:166-186
// score_pairs -> CudaPairHMM.score, :105-159) takes a list of (read,
// qualities, haplotype) triples, validates it in Python (:25-40) and packs it
// per bucket (:64-78); its CPU batch path (cpu_batch.py:44-62) dedupes the
// jobs and sorts them by length before calling the native kernels.  Here that
// host work is native: the Python layer hands over pointer arrays into its
// own objects (the batch_hmm.cpp:192 calling convention) and this file
//
//  1. checks every distinct read and haplotype for uppercase ACGTN (the
//     reference's "Uppercase DNA required" rule; qualities are bytes already);
//  2. gives identical reads (same bases and qualities) and identical
//     haplotypes one id each, first by pointer (a caller passes the same
//     object with every haplotype of a read) and then by content;
//  3. drops repeated (read, haplotype) pairs and regroups the reads into
//     regions: reads that ask for the same set of haplotypes form one region,
//     which is the shape the two-read packed kernels and the shared-prefix
//     schedule need (a caller's pair list is usually reads x haplotypes of its
//     active regions, concatenated);
//  4. scores the region batch with vd_forward and scatters the results back
//     to the input order.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/vardepth_pairhmm.h"
#include "pairhmm_launch.h"

namespace vd {
namespace {

// every byte one of A, C, G, T, N (comparisons the compiler vectorises)
bool is_dna(const unsigned char* p, int n) {
  unsigned char bad = 0;
  for (int i = 0; i < n; ++i) {
    const unsigned char c = p[i];
    bad |= (unsigned char)((c != 'A') & (c != 'C') & (c != 'G') & (c != 'T') & (c != 'N'));
  }
  return bad == 0;
}

// 64-bit hash of a byte string (multiply-xorshift over 8-byte words).  Long
// strings are sampled at up to 16 words spread over their length: equal
// hashes are always confirmed by a full comparison, so the sample only has to
// tell most different strings apart.
uint64_t hash_bytes(const unsigned char* p, int n, uint64_t h) {
  constexpr uint64_t kMul = 0x9e3779b97f4a7c15ull;
  const int words = n / 8;
  const int step = words > 16 ? words / 16 : 1;
  for (int k = 0; k < words; k += step) {
    uint64_t w;
    std::memcpy(&w, p + 8 * k, 8);
    h = (h ^ w) * kMul;
    h ^= h >> 29;
  }
  uint64_t w = 0;
  if (n > 8 * words) std::memcpy(&w, p + 8 * words, (size_t)(n - 8 * words));
  else if (n >= 8) std::memcpy(&w, p + n - 8, 8);
  h = (h ^ w ^ ((uint64_t)n << 56)) * kMul;
  return h ^ (h >> 32);
}

// Open-addressing table of (hash, id) with linear probing; grows at half load.
class IdTable {
 public:
  // the id stored under hash h for which same(id) holds, else -1
  template <typename Same>
  int32_t find(uint64_t h, Same&& same) const {
    if (slots_.empty()) return -1;
    for (size_t i = (size_t)h & mask_;; i = (i + 1) & mask_) {
      const Entry& e = slots_[i];
      if (e.id < 0) return -1;
      if (e.h == h && same(e.id)) return e.id;
    }
  }
  void insert(uint64_t h, int32_t id) {
    if (2 * (used_ + 1) > slots_.size()) grow();
    size_t i = (size_t)h & mask_;
    while (slots_[i].id >= 0) i = (i + 1) & mask_;
    slots_[i] = Entry{h, id};
    ++used_;
  }

 private:
  struct Entry {
    uint64_t h = 0;
    int32_t id = -1;
  };
  void grow() {
    std::vector<Entry> old;
    old.swap(slots_);
    slots_.assign(old.empty() ? 1024 : 2 * old.size(), Entry{});
    mask_ = slots_.size() - 1;
    used_ = 0;
    for (const Entry& e : old)
      if (e.id >= 0) insert(e.h, e.id);
  }
  std::vector<Entry> slots_;
  size_t mask_ = 0, used_ = 0;
};

// Distinct byte strings (a read is its bases and qualities, a haplotype its
// bases): ids in order of first appearance.  A direct-mapped cache of recent
// pointers answers repeats of the same object (a caller passes each read's
// objects with every haplotype, and the same few haplotype objects over and
// over); a new pointer is checked for ACGTN and looked up by content.
class Interner {
 public:
  std::vector<const unsigned char*> bases, quals;
  std::vector<int> len;

  // track_pointers: keep every pointer seen (haplotype objects recur all over
  // a pair list); without it a pointer evicted from the cache is looked up by
  // content again (a read's object recurs only in its own run of pairs)
  explicit Interner(bool track_pointers) : track_(track_pointers) {}

  // id of (b, q, n); -1 when the bases are not uppercase ACGTN
  int32_t id(const unsigned char* b, const unsigned char* q, int n) {
    uint64_t hp = ((uint64_t)(uintptr_t)b * 0x9e3779b97f4a7c15ull) ^ ((uint64_t)(uintptr_t)q * 0xc2b2ae3d27d4eb4full) ^
                  (uint64_t)n;
    hp ^= hp >> 29;
    Slot& c = cache_[hp & (kCache - 1)];
    if (c.id >= 0 && c.b == b && c.q == q && c.n == n) return c.id;
    if (track_) {  // a pointer seen before, evicted from the cache
      const int32_t e = by_ptr_.find(hp, [&](int32_t k) {
        const Slot& x = ptrs_[(size_t)k];
        return x.b == b && x.q == q && x.n == n;
      });
      if (e >= 0) {
        c = ptrs_[(size_t)e];
        return c.id;
      }
    }
    const int32_t r = by_content(b, q, n);
    if (r < 0) return -1;
    c = Slot{b, q, n, r};
    if (track_) {
      by_ptr_.insert(hp, (int32_t)ptrs_.size());
      ptrs_.push_back(c);
    }
    return r;
  }

 private:
  int32_t by_content(const unsigned char* b, const unsigned char* q, int n) {
    if (!is_dna(b, n)) return -1;
    uint64_t h = n ? hash_bytes(b, n, 0x51ed27e5u) : 0x51ed27e5u;
    if (q && n) h = hash_bytes(q, n, h);
    int32_t r = by_content_.find(h, [&](int32_t j) {
      return len[(size_t)j] == n && (n == 0 || (std::memcmp(bases[(size_t)j], b, (size_t)n) == 0 &&
                                                (!q || std::memcmp(quals[(size_t)j], q, (size_t)n) == 0)));
    });
    if (r < 0) {
      r = (int32_t)len.size();
      bases.push_back(b);
      quals.push_back(q);
      len.push_back(n);
      by_content_.insert(h, r);
    }
    return r;
  }

  struct Slot {
    const unsigned char* b = nullptr;
    const unsigned char* q = nullptr;
    int n = -1;
    int32_t id = -1;
  };
  static constexpr size_t kCache = 4096;
  std::vector<Slot> cache_ = std::vector<Slot>(kCache);
  bool track_;
  std::vector<Slot> ptrs_;  // every distinct (pointer, length) seen, with its id
  IdTable by_ptr_, by_content_;
};

// The regrouped batch: regions of reads that ask for the same haplotype set.
struct PairListPlan {
  Interner reads{false}, haps{true};
  std::vector<int32_t> pair_read, pair_hap, pair_region;
  std::vector<int64_t> pair_slot;          // output slot of each input pair in the region batch
  std::vector<int32_t> read_region;        // region of each distinct read
  std::vector<int64_t> region_read_off{0}; // into region_reads
  std::vector<int32_t> region_reads;       // distinct reads, region by region
  std::vector<int64_t> region_hap_off{0};  // into region_haps
  std::vector<int32_t> region_haps;        // distinct haplotypes (sorted ids), region by region
  std::vector<int64_t> region_out_off{0};
};

int build_plan(const char* const* rs, const unsigned char* const* qs, const int* rn, const char* const* hs,
               const int* hn, int64_t count, PairListPlan& pl) {
  pl.pair_read.resize((size_t)count);
  pl.pair_hap.resize((size_t)count);
  for (int64_t p = 0; p < count; ++p) {
    const int n = rn[p], m = hn[p];
    if (n < 0 || m < 0) return report_error(VD_EINVAL, ("negative length at pair " + std::to_string(p)).c_str());
    if ((n > 0 && (!rs[p] || !qs[p])) || (m > 0 && !hs[p]))
      return report_error(VD_EINVAL, ("NULL sequence at pair " + std::to_string(p)).c_str());
    const int32_t r = pl.reads.id((const unsigned char*)rs[p], qs[p], n);
    const int32_t h = pl.haps.id((const unsigned char*)hs[p], nullptr, m);
    if (r < 0 || h < 0) return report_error(VD_EINVAL, "Uppercase DNA required");
    pl.pair_read[(size_t)p] = r;
    pl.pair_hap[(size_t)p] = h;
  }
  // each read's distinct haplotypes (counting sort by read, then sort + unique)
  const int64_t nr = (int64_t)pl.reads.len.size();
  std::vector<int64_t> start((size_t)nr + 1, 0);
  for (int64_t p = 0; p < count; ++p) ++start[(size_t)pl.pair_read[(size_t)p] + 1];
  for (int64_t r = 0; r < nr; ++r) start[(size_t)r + 1] += start[(size_t)r];
  std::vector<int32_t> hl((size_t)count);
  {
    std::vector<int64_t> fill(start.begin(), start.end() - 1);
    for (int64_t p = 0; p < count; ++p) hl[(size_t)fill[(size_t)pl.pair_read[(size_t)p]]++] = pl.pair_hap[(size_t)p];
  }
  std::vector<int64_t> ustart((size_t)nr + 1, 0);  // unique lists, compacted in place
  int64_t w = 0;
  for (int64_t r = 0; r < nr; ++r) {
    auto b = hl.begin() + start[(size_t)r], e = hl.begin() + start[(size_t)r + 1];
    std::sort(b, e);
    e = std::unique(b, e);
    ustart[(size_t)r] = w;
    for (auto it = b; it != e; ++it) hl[(size_t)w++] = *it;
  }
  ustart[(size_t)nr] = w;
  // reads with equal lists form a region (regions in order of their first read)
  pl.read_region.assign((size_t)nr, -1);
  IdTable by_list;
  std::vector<int32_t> region_first;  // a read of each region (its list is the region's)
  std::vector<std::vector<int32_t>> members;
  int32_t prev_g = -1;
  for (int64_t r = 0; r < nr; ++r) {
    const int32_t* lb = hl.data() + ustart[(size_t)r];
    const int64_t ln = ustart[(size_t)r + 1] - ustart[(size_t)r];
    auto same_list = [&](int32_t g) {
      const int32_t f = region_first[(size_t)g];
      return ustart[(size_t)f + 1] - ustart[(size_t)f] == ln && std::equal(lb, lb + ln, hl.data() + ustart[(size_t)f]);
    };
    // consecutive reads usually belong to the same region
    int32_t g = (prev_g >= 0 && same_list(prev_g)) ? prev_g : -1;
    if (g < 0) {
      const uint64_t h = hash_bytes(reinterpret_cast<const unsigned char*>(lb), (int)(ln * 4), 0x2545f491u);
      g = by_list.find(h, same_list);
      if (g < 0) {
        g = (int32_t)region_first.size();
        region_first.push_back((int32_t)r);
        members.emplace_back();
        by_list.insert(h, g);
      }
    }
    prev_g = g;
    pl.read_region[(size_t)r] = g;
    members[(size_t)g].push_back((int32_t)r);
  }
  // region layout and each read's position in its region
  const size_t ng = region_first.size();
  std::vector<int32_t> local((size_t)nr, 0);
  for (size_t g = 0; g < ng; ++g) {
    for (size_t i = 0; i < members[g].size(); ++i) {
      local[(size_t)members[g][i]] = (int32_t)i;
      pl.region_reads.push_back(members[g][i]);
    }
    pl.region_read_off.push_back((int64_t)pl.region_reads.size());
    const int32_t f = region_first[g];
    pl.region_haps.insert(pl.region_haps.end(), hl.begin() + ustart[(size_t)f], hl.begin() + ustart[(size_t)f + 1]);
    pl.region_hap_off.push_back((int64_t)pl.region_haps.size());
    const int64_t nh = ustart[(size_t)f + 1] - ustart[(size_t)f];
    pl.region_out_off.push_back(pl.region_out_off.back() + (int64_t)members[g].size() * nh);
  }
  // output slot of every input pair
  pl.pair_region.resize((size_t)count);
  pl.pair_slot.resize((size_t)count);
  for (int64_t p = 0; p < count; ++p) {
    const int32_t r = pl.pair_read[(size_t)p];
    const int32_t g = pl.read_region[(size_t)r];
    const int32_t* hb = pl.region_haps.data() + pl.region_hap_off[(size_t)g];
    const int64_t nh = pl.region_hap_off[(size_t)g + 1] - pl.region_hap_off[(size_t)g];
    const int64_t j = std::lower_bound(hb, hb + nh, pl.pair_hap[(size_t)p]) - hb;
    pl.pair_region[(size_t)p] = g;
    pl.pair_slot[(size_t)p] = pl.region_out_off[(size_t)g] + (int64_t)local[(size_t)r] * nh + j;
  }
  return VD_OK;
}

// A byte buffer that grows without zero-filling and keeps its pages.
struct Bytes {
  std::unique_ptr<unsigned char[]> p;
  size_t cap = 0;
  unsigned char* reserve(size_t n) {
    if (n > cap) {
      p.reset(new unsigned char[n]);
      cap = n;
    }
    return p.get();
  }
};

// The packed buffers of the region batch; one set per calling thread, reused
// from call to call (like the reference's thread_local scratch,
// batch_hmm.cpp:21), so repeated calls do not fault fresh pages in.
struct RegionBatch {
  Bytes rb, rq, hb;
  std::vector<int64_t> roff, hoff, rr, hr;
  vd_batch batch{};
};

void pack_regions(const PairListPlan& pl, RegionBatch& rb) {
  const size_t ng = pl.region_read_off.size() - 1;
  int64_t rbytes = 0, hbytes = 0;
  for (int32_t r : pl.region_reads) rbytes += pl.reads.len[(size_t)r];
  for (int32_t h : pl.region_haps) hbytes += pl.haps.len[(size_t)h];
  unsigned char* const rbp = rb.rb.reserve((size_t)rbytes + 1);
  unsigned char* const rqp = rb.rq.reserve((size_t)rbytes + 1);
  unsigned char* const hbp = rb.hb.reserve((size_t)hbytes + 1);
  rb.roff.assign(1, 0);
  rb.hoff.assign(1, 0);
  rb.rr.assign(1, 0);
  rb.hr.assign(1, 0);
  rb.roff.reserve(pl.region_reads.size() + 1);
  rb.hoff.reserve(pl.region_haps.size() + 1);
  int64_t o = 0;
  for (int32_t r : pl.region_reads) {
    const int n = pl.reads.len[(size_t)r];
    if (n) {
      std::memcpy(rbp + o, pl.reads.bases[(size_t)r], (size_t)n);
      std::memcpy(rqp + o, pl.reads.quals[(size_t)r], (size_t)n);
    }
    o += n;
    rb.roff.push_back(o);
  }
  o = 0;
  for (int32_t h : pl.region_haps) {
    const int m = pl.haps.len[(size_t)h];
    if (m) std::memcpy(hbp + o, pl.haps.bases[(size_t)h], (size_t)m);
    o += m;
    rb.hoff.push_back(o);
  }
  for (size_t g = 0; g < ng; ++g) {
    rb.rr.push_back(pl.region_read_off[g + 1]);
    rb.hr.push_back(pl.region_hap_off[g + 1]);
  }
  vd_batch& b = rb.batch;
  b.read_bases = rbp;
  b.read_quals = rqp;
  b.read_off = rb.roff.data();
  b.n_reads = (int64_t)rb.roff.size() - 1;
  b.hap_bases = hbp;
  b.hap_off = rb.hoff.data();
  b.n_haps = (int64_t)rb.hoff.size() - 1;
  b.region_read_off = rb.rr.data();
  b.region_hap_off = rb.hr.data();
  b.n_regions = (int64_t)ng;
}

int check_arrays(const void* reads, const void* quals, const int* rn, const void* haps, const int* hn,
                 int64_t count) {
  if (count < 0) return report_error(VD_EINVAL, "count < 0");
  if (count > 0 && (!reads || !quals || !rn || !haps || !hn)) return report_error(VD_EINVAL, "NULL argument");
  return VD_OK;
}

}  // namespace
}  // namespace vd

using namespace vd;

extern "C" int vd_pair_list_plan(const char* const* reads, const unsigned char* const* quals, const int* rn,
                                 const char* const* haps, const int* hn, int64_t count, int64_t* counts,
                                 int32_t* pair_read, int32_t* pair_hap, int32_t* pair_region, int64_t* pair_slot) {
  int rc = check_arrays(reads, quals, rn, haps, hn, count);
  if (rc) return rc;
  if (!counts) return report_error(VD_EINVAL, "counts is NULL");
  PairListPlan pl;
  if ((rc = build_plan(reads, quals, rn, haps, hn, count, pl))) return rc;
  counts[0] = (int64_t)pl.reads.len.size();
  counts[1] = (int64_t)pl.haps.len.size();
  counts[2] = (int64_t)pl.region_read_off.size() - 1;
  counts[3] = pl.region_out_off.back();
  const size_t bytes = (size_t)count;
  if (pair_read && count) std::memcpy(pair_read, pl.pair_read.data(), bytes * 4);
  if (pair_hap && count) std::memcpy(pair_hap, pl.pair_hap.data(), bytes * 4);
  if (pair_region && count) std::memcpy(pair_region, pl.pair_region.data(), bytes * 4);
  if (pair_slot && count) std::memcpy(pair_slot, pl.pair_slot.data(), bytes * 8);
  return VD_OK;
}

extern "C" int vd_score_pair_list(vd_engine* engine, const char* const* reads, const unsigned char* const* quals,
                                  const int* rn, const char* const* haps, const int* hn, int64_t count,
                                  const vd_params* params, double* out, vd_stats* stats) {
  if (!engine) return report_error(VD_EINVAL, "engine is NULL");
  if (!params) return report_error(VD_EINVAL, "params is NULL");
  int rc = check_arrays(reads, quals, rn, haps, hn, count);
  if (rc) return rc;
  if (count > 0 && !out) return report_error(VD_EINVAL, "out is NULL");
  vd_stats s{};
  if (count == 0) {
    if (stats) *stats = s;
    return VD_OK;
  }
  const auto t0 = std::chrono::steady_clock::now();
  PairListPlan pl;
  if ((rc = build_plan(reads, quals, rn, haps, hn, count, pl))) return rc;
  thread_local RegionBatch rb;
  pack_regions(pl, rb);
  thread_local std::vector<double> region_out;
  region_out.resize((size_t)pl.region_out_off.back());
  const double plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if ((rc = vd_forward(engine, &rb.batch, params, region_out.data(), &s))) return rc;
  for (int64_t p = 0; p < count; ++p) out[p] = region_out[(size_t)pl.pair_slot[(size_t)p]];
  s.pairs = count;
  s.host_ms += plan_ms;
  s.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (stats) *stats = s;
  return VD_OK;
}
