// Long reads (more rows than one 256-row strip), FP32, semiglobal: one warp
// runs one read against up to kLongGroupMax haplotypes of its region, TWO at
// a time.
//
// The read's rows are packed as float2 over the two haplotypes of a pair (x:
// the first, y: the second), so every FMA serves both (fma.rn.f32x2) and the
// read's per-row constants, its strip count and its strip bookkeeping are
// shared: the halves always have the same number of strips, which two reads
// of different lengths would not.  A region's haplotypes differ by a few
// small edits, so their lengths nearly agree and the shorter one idles for a
// few columns at most.
//
// Range.  An error-rich read (8% errors at reported Q30) loses about one bit
// per row along its best path, far more over a 256-row strip than FP32 holds,
// so lane L scales everything it takes from above by 2^k_L.  A boost on a
// lane's inputs scales the lane's rows and everything below by an exact power
// of two, so the rows keep the one-sided emission (a match costs no multiply)
// and the boosts are undone exactly in the final exponent.  The first pair of
// an item spreads each strip's predicted decay (the read's mean rate so far
// times the strip's rows) evenly over the lanes; a strip whose bottom leaves
// 2^-60 .. 2^60, or a lane whose bottom-row maximum leaves 2^-90 .. 2^90, is
// run again with each lane's measured decay (its input boundary is kept: the
// warp's slot holds two boundary buffers, one read and one written).  The
// pairs after the first start each strip from the first pair's measured lane
// decays, since the read's errors sit at the same rows against every
// haplotype.  The first strip starts from 2^60.  A strip's boundary is stored
// as computed and brought to 2^0 by an exact power of two as the next strip
// loads it.  A pair still out of range after kLongTries runs of a strip, or
// decaying faster than kLongMaxRate bits per row, goes to the drift and FP64
// tiers.
//
// Every choice above depends on the item's own data (a first pair's boosts on
// that pair alone, per half; a re-run caused by the other half recomputes this
// half's strip bit for bit; the later pairs' on the first pair's
// measurements), and the final log is taken as ln f + (e - E) ln 2 with the
// sum z = f 2^e, so the bits do not depend on which powers of two the boosts
// took.  The plain schedule forms the same items and gives the same bits.
#pragma once
#include "pairhmm_kernel.cuh"

namespace vd {

constexpr int kLongTries = 6;       // runs of one strip before a half gives up
// A strip bottom must end in 2^-60 .. 2^60: the cells that carry the mass lie
// within a few dozen binary orders below the bottom's maximum, and they must
// stay far above 2^-126, where the packed f32x2 arithmetic loses them (with
// bottoms allowed down to 2^-100 the error reached 8e-4 log10 on 8%-error
// 7 kb reads, down to 2^-120 0.1; at 2^-60 it stays at the FP32 rounding level)
constexpr int kLongFloor = -60;
constexpr int kLongCeil = 60;
constexpr int kLongStart = 60;      // the first strip's input, 2^60 (binary orders)

template <int R>
struct LongRows {
  uint32_t rb[R];        // read bases (kNeverBase for rows past the read)
  float miss[R];         // mismatch factor of rows 1 .. R-1 (the same for both halves)
  float2 hit0, miss0;    // row 0's match and mismatch factors times the lane's boost, per half
  float2 K[R], X[R];     // k1 f_i and (x/4) f_i (alpha f_n on the last row), both halves
                         // (row 0's times the lane's boost)
  float2 W[R], s[R];     // om of the next column and s of the column finished last
};

// The lane's boost 2^k multiplies every term that row 0 takes from above (the
// diagonal s and the vertical u), so it is folded into row 0's factors once
// per strip instead of into the two inputs at every step: the products are
// the same bits (a power of two times a normal float is exact) and the
// vertical chain through the lane's rows is one multiply shorter.
template <int R>
__device__ __forceinline__ void boost_row0(LongRows<R>& w, const float2 bf) {
  w.hit0 = bf;
  w.miss0 = make_float2(w.miss[0] * bf.x, w.miss[0] * bf.y);
  w.K[0] = __fmul2_rn(w.K[0], bf);
  w.X[0] = __fmul2_rn(w.X[0], bf);
}

template <int R>
__device__ __forceinline__ void column_long(LongRows<R>& w, uint32_t hbx, uint32_t hby, float2 s_top, float2 u_top,
                                            float2 k2, float2 x, float2& u_bot) {
  float2 s_above = s_top;
  float2 nu = u_top;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    float2 mu_new;
    if (r == 0) {
      const float fx = w.rb[0] == hbx ? w.hit0.x : w.miss0.x;
      const float fy = w.rb[0] == hby ? w.hit0.y : w.miss0.y;
      mu_new = __fmul2_rn(s_above, make_float2(fx, fy));
    } else {
      mu_new = s_above;
      mul_if_ne(mu_new.x, w.rb[r], hbx, w.miss[r]);
      mul_if_ne(mu_new.y, w.rb[r], hby, w.miss[r]);
    }
    const float2 om_new = w.W[r];
    const float2 u_new = __ffma2_rn(w.X[r], nu, mu_new);
    const float2 s_new = __ffma2_rn(k2, om_new, __ffma2_rn(w.K[r], nu, mu_new));
    s_above = w.s[r];
    w.W[r] = __ffma2_rn(x, om_new, mu_new);
    w.s[r] = s_new;
    nu = u_new;
  }
  u_bot = nu;
}

// exponent of a boundary maximum or final sum, +-1024 for inf/NaN and zero
__device__ __forceinline__ int long_exponent(float v) {
  return (v != v || v >= HUGE_VALF) ? 1024 : (v > 0.f ? ilogbf(v) : -1024);
}
__device__ __forceinline__ int long_exponent(double v) {
  return (v != v || v >= HUGE_VAL) ? 1024 : (v > 0.0 ? ilogb(v) : -1024);
}

// One half's lane boosts after a run of a strip that left the window.  Lane
// L measured the maximum of its bottom row (exponent lg_L, +-1024 for inf or
// zero); with its input at 2^lg_{L-1} (lane 0: the strip's input, 2^in0) and
// boost k_L, its rows decayed by d_L = k_L + lg_{L-1} - lg_L bits, and the
// boost d_L (lane 0: d_0 - in0) brings its bottom to 2^0 wherever in the
// strip the read's errors sit.  The first lane whose bottom under- or
// overflowed moves by the bound that shows (a nonzero float lies above
// 2^-149, a finite one below 2^128), and the lanes below it, whose inputs
// are unknown, take the mean rate of the lanes above.  Shares stay within
// -96 .. 120 bits, where 2^k times every row factor is a normal float.
__device__ __forceinline__ int relane(const int kl, const float lm, const int used, const int lrows, const int in0,
                                      const int lane) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lg = lane < used ? long_exponent(lm) : 0;
  int in = __shfl_up_sync(FULL, lg, 1);
  if (lane == 0) in = in0;
  const int tgt = lane == 0 ? in0 : 0;  // the input the next run's lane sees
  const bool measured = lg > -1024 && lg < 1024;
  const unsigned bad = __ballot_sync(FULL, lane < used && !measured);
  const int first_bad = bad ? __ffs(bad) - 1 : kWarp;
  const bool valid = lane < used && lane < first_bad;
  const int d = valid ? kl + in - lg : 0;
  int sum_d = d, sum_r = valid ? lrows : 0;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    sum_d += __shfl_xor_sync(FULL, sum_d, o);
    sum_r += __shfl_xor_sync(FULL, sum_r, o);
  }
  if (lane >= used) return 0;
  int k = kl;
  if (valid) {
    k = d - tgt;
  } else {
    if (sum_r > 0) k = (int)((long long)sum_d * lrows / sum_r) - tgt;
    if (lane == first_bad) k = lg == -1024 ? max(k, kl + in + 149 - tgt) : min(k, kl + in - 128 - tgt);
  }
  return max(-96, min(120, k));
}

// Strips of a read whose per-lane decays the first pair of an item records
// (longer reads predict the rest from the mean rate), and the window a lane's
// bottom-row maximum must end in for a run to be kept.
constexpr int kLongProfStrips = 80;
// Boost bits per row a strip may take (an error-rich read at 8% errors and
// reported Q30 takes about one; a random read against a random haplotype
// four to five)
constexpr int kLongMaxRate = 4;
constexpr int kLongLaneFloor = -90;
constexpr int kLongLaneCeil = 90;

// One work item: read w.read against haplotypes hap_begin .. hap_begin +
// nhap - 1 (nhap <= kLongGroupMax), two at a time; outputs out_begin + k.
// `scratch` is the warp's slot: 2 * half float4 boundary records (half >= the
// longest haplotype + 1); `ring` and `oring` 32 float4 each of shared memory
// per warp (the boundary read, the boundary written); `prof` the warp's
// kLongProfStrips x 32 per-lane decays.
template <int R>
__device__ __noinline__ void process_long(const BatchView bv, const QueueView qv, const WorkItem w,
                                          const Tables<float>* __restrict__ tb, const Scalars<float> sc,
                                          const int lane, float4* __restrict__ scratch, float4* __restrict__ ring,
                                          float4* __restrict__ oring, short* __restrict__ prof) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr double kLn2 = 0.6931471805599453094;
  constexpr int SR = kWarp * R;
  const int64_t roff = bv.read_off[w.read];
  const int n = (int)(bv.read_off[w.read + 1] - roff);
  const uint8_t* __restrict__ rbase = bv.read_bases + roff;
  const uint8_t* __restrict__ rqual = bv.read_quals + roff;
  const int nstrips = (n + SR - 1) / SR;
  const long long half = qv.scratch_stride / 2;

  double lnN = 0.0;
  for (int i = lane; i < n; i += kWarp) lnN += tb->lnN[rqual[i]];
#pragma unroll
  for (int o = 16; o; o >>= 1) lnN += __shfl_xor_sync(FULL, lnN, o);
  const float A = tb->A[rqual[n - 1]];
  const float2 k2 = make_float2(sc.k2, sc.k2), x = make_float2(sc.x, sc.x);
  const float c0 = sc.c;

  // the item's first pair records each strip's per-lane decays (of its first
  // half while that is in play, else its second); the pairs after it start a
  // recorded strip from them and the rest from the mean rate
  int prof_len = 0;
  // every lane holding read rows ended its bottom row in the lane window
  auto lanes_in_window = [&](const float lm, const int used) -> bool {
    const int lg = long_exponent(lm);
    return __all_sync(FULL, lane >= used || (lg >= kLongLaneFloor && lg < kLongLaneCeil));
  };

  for (int g = 0; g < w.nhap; g += 2) {
    // the pair in hand
    const bool two = g + 1 < w.nhap;
    const int64_t h1 = w.hap_begin + g, h2 = two ? h1 + 1 : h1;
    const int64_t ho1 = bv.hap_off[h1], ho2 = bv.hap_off[h2];
    const int m1 = (int)(bv.hap_off[h1 + 1] - ho1), m2 = (int)(bv.hap_off[h2 + 1] - ho2);
    const uint8_t* __restrict__ hp1 = bv.hap_bases + ho1 - 1;  // hp[j] = base of column j >= 1
    const uint8_t* __restrict__ hp2 = bv.hap_bases + ho2 - 1;
    const int M = max(m1, m2);

    // per half: boost bits of the current strip, total exponent, still in play
    int Bx = 0, By = 0, Ex = 0, Ey = 0;
    // decay measured over the strips done so far (bits, rows): the next strip's
    // boost is this mean rate times its rows.  A single strip's decay scatters
    // by tens of bits around the read's rate (the number of errors in 256 rows),
    // so the mean predicts the next strip about sqrt(2) times better than the
    // last strip alone, and fewer strips run twice
    int Dx = 0, Dy = 0, Nrows = 0;
    bool okx = true, oky = two;
    int inx = 0, iny = 0;        // shifts that bring the boundary above to 2^0, per half
    int lgx = 0, lgy = 0;        // bottom exponents of the last run
    double zx = 0.0, zy = 0.0;   // final sums (last strip, lane 31)
    int klx = 0, kly = 0;        // this lane's share of the strip's boost, per half
    float lmx = 0.f, lmy = 0.f;  // this lane's bottom-row maxima in the last run

    // One run of strip `strip` with Bx / By boost bits; reads boundary buffer
    // src_half, writes the other.  Sets lgx / lgy (bottom maximum or final sum).
    auto run_strip = [&](const int strip, const bool last) {
      const int i0 = strip * SR;
      const int ns = min(SR, n - i0);           // read rows of the strip
      const int lanes_used = (ns + R - 1) / R;  // lanes holding read rows
      LongRows<R> rw;
  #pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = i0 + lane * R + r;
        if (i < n) {
          const unsigned q = rqual[i];
          rw.rb[r] = rbase[i];
          rw.miss[r] = tb->miss[q];
          const float K = tb->K[q], X = (i == n - 1) ? A : tb->X[q];
          rw.K[r] = make_float2(K, K);
          rw.X[r] = make_float2(X, X);
        } else {  // past the read: pass u down the column
          rw.rb[r] = kNeverBase;
          rw.miss[r] = 0.f;
          rw.K[r] = make_float2(0.f, 0.f);
          rw.X[r] = make_float2(1.f, 1.f);
        }
        rw.W[r] = make_float2(0.f, 0.f);
        rw.s[r] = make_float2(0.f, 0.f);
      }
      // lane L's share of the boost: floor((L+1) B / lanes) - floor(L B / lanes)
      // over the lanes holding read rows; the first strip's input starts at 2^kLongStart
      // (|B| <= 4 ns keeps every share within +-4R, far inside the float exponent range)
      boost_row0(rw, make_float2(pow2T(klx, 0.f), pow2T(kly, 0.f)));
      const float cin = c0 * pow2T(kLongStart, 0.f);  // the first strip's row-0 value
      float4* const src = scratch + (long long)(strip & 1) * half;
      float4* const dst = scratch + (long long)((strip + 1) & 1) * half;
      // the boundary above is stored as written (its maximum at 2^lg); it is
      // brought to 2^0 as it is loaded, by 2^-lg per half
      const float fsx = pow2T(inx, 0.f), fsy = pow2T(iny, 0.f);

      float2 s_top = make_float2(0.f, 0.f), u_bot = make_float2(0.f, 0.f), acc32 = make_float2(0.f, 0.f);
      double accx = 0.0, accy = 0.0;
      float bmx = 0.f, bmy = 0.f;
      float2 lm = make_float2(0.f, 0.f);  // this lane's bottom-row maxima
      const bool lane0 = lane == 0;
      // boundary records of the strip above, staged through the warp's ring:
      // every 32 steps each lane loads one record of the next 32 columns, and
      // at every step all lanes read the record of lane 0's column (a broadcast)
      float4 nxt = make_float4(0.f, 0.f, 0.f, 0.f);
      auto load_window = [&](int base) -> float4 {
        const int p = base + lane;
        if (strip == 0 || p > M) return make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 v = src[p];
        return make_float4(v.x * fsx, v.y * fsx, v.z * fsy, v.w * fsy);
      };
      auto stage_window = [&](int t) {
        __syncwarp();
        ring[lane] = nxt;
        __syncwarp();
        nxt = load_window(t + kWarp);
      };
      // this strip's bottom rows: lane 31 lays each column's record into the
      // warp's out-ring, and every 32 columns the warp writes them to the
      // boundary buffer in one coalesced store and folds them into the maxima
      int flushed = 0;  // columns below this are in the boundary buffer
      auto flush_out = [&](int count) {
        __syncwarp();
        if (lane < count) {
          const int p = flushed + lane;
          const float4 rec = oring[lane];
          dst[p] = rec;
          if (p <= m1) bmx = fmaxf(bmx, fmaxf(rec.x, rec.y));
          if (p <= m2) bmy = fmaxf(bmy, fmaxf(rec.z, rec.w));
        }
        __syncwarp();
        flushed += count;
      };
      // lane 31 moves its FP32 row sums into FP64 after its columns 8r+7
      auto flush_acc = [&]() {
        accx += (double)acc32.x;
        accy += (double)acc32.y;
        acc32 = make_float2(0.f, 0.f);
      };
      const float2 cin2 = make_float2(cin, cin);
      // one step; STEADY: every lane inside both haplotypes at a column >= 1
      auto step = [&](auto steady_tag, const int t) {
        constexpr bool STEADY = decltype(steady_tag)::value;
        const int p = t - lane;  // this lane's column
        // lane 0's boundary record is loaded before the shuffles, so its
        // latency runs beside theirs rather than after them on the chain
        // (20,000 mixed-length regions: 1,003 against 1,053 ms per step)
        float2 in_s = cin2, in_u = cin2;
        if (strip > 0) {
          const float4 rec = ring[t & (kWarp - 1)];
          in_s = make_float2(rec.x, rec.z);
          in_u = make_float2(rec.y, rec.w);
        }
        float2 u_in = shfl_up2(u_bot);
        float2 s_in = shfl_up2(rw.s[R - 1]);
        u_in = lane0 ? in_u : u_in;
        s_in = lane0 ? in_s : s_in;
        bool inside = true;
        uint32_t hbx, hby;
        if (STEADY) {
          hbx = hp1[p];
          hby = hp2[p];
        } else {
          // column 0 has no base (kNeverBase never matches); past a haplotype's
          // end its half reads that haplotype's last base (its columns are not used)
          inside = p >= 0 && p <= M;
          hbx = (inside && p > 0) ? (uint32_t)hp1[min(p, m1)] : kNeverBase;
          hby = (inside && p > 0) ? (uint32_t)hp2[min(p, m2)] : kNeverBase;
        }
        column_long<R>(rw, hbx, hby, (STEADY || p > 0) ? s_top : make_float2(0.f, 0.f), u_in, k2, x, u_bot);
        if (STEADY) {
          lm.x = fmaxf(lm.x, u_bot.x);
          lm.y = fmaxf(lm.y, u_bot.y);
        } else {
          if (inside && p <= m1) lm.x = fmaxf(lm.x, u_bot.x);
          if (inside && p <= m2) lm.y = fmaxf(lm.y, u_bot.y);
        }
        if (!STEADY && p <= 0) {
          // column 0 (and the lanes not started yet): no diagonal, no deletions
  #pragma unroll
          for (int r = 0; r < R; ++r) rw.W[r] = make_float2(0.f, 0.f);
        }
        s_top = s_in;
        if (last) {
          // the final row sums (lane 31's are the ones used)
          if (STEADY) {
            acc32 = __fadd2_rn(acc32, u_bot);
          } else if (lane == kWarp - 1 && inside) {
            if (p <= m1) acc32.x += u_bot.x;
            if (p <= m2) acc32.y += u_bot.y;
            if ((p & 7) == 7) flush_acc();
          }
        } else if (lane == kWarp - 1 && inside) {
          oring[p & (kWarp - 1)] = make_float4(rw.s[R - 1].x, u_bot.x, rw.s[R - 1].y, u_bot.y);
        }
      };
      // the out-ring is full when lane 31 has finished column flushed + 31
      auto maybe_flush = [&](int t) {
        if (!last && t - (kWarp - 1) == flushed + kWarp - 1) flush_out(kWarp);
      };

      nxt = load_window(0);
      const int steps = M + 1 + (kWarp - 1);
      // steady steps: every lane at a column in 1 .. min(m1, m2)
      const int t_lo = kWarp, t_hi = min(m1, m2) + 1;
      int t = 0;
      for (; t < steps && (t < t_lo || (t < t_hi && (t & 7) != 0)); ++t) {
        if ((t & (kWarp - 1)) == 0) stage_window(t);
        step(std::false_type{}, t);
        maybe_flush(t);
      }
      // blocks of 8 steps start at a multiple of 8, so lane 31's columns 8r+7
      // fall at the block's step 6 and its out-ring fills at step 6 of every
      // fourth block
      for (; t + 8 <= t_hi; t += 8) {
        if ((t & (kWarp - 1)) == 0) stage_window(t);
  #pragma unroll
        for (int u = 0; u < 8; ++u) {
          step(std::true_type{}, t + u);
          if (u == 6) {
            if (last) flush_acc();
            else maybe_flush(t + u);
          }
        }
      }
      for (; t < steps; ++t) {
        if ((t & (kWarp - 1)) == 0) stage_window(t);
        step(std::false_type{}, t);
        maybe_flush(t);
      }
      if (!last && flushed <= M) flush_out(M + 1 - flushed);
      if (!last) {
  #pragma unroll
        for (int o = 16; o; o >>= 1) {
          bmx = fmaxf(bmx, __shfl_xor_sync(FULL, bmx, o));
          bmy = fmaxf(bmy, __shfl_xor_sync(FULL, bmy, o));
        }
      }
      __syncwarp();
      if (last) {
        zx = __shfl_sync(FULL, accx + (double)acc32.x, kWarp - 1);
        zy = __shfl_sync(FULL, accy + (double)acc32.y, kWarp - 1);
        lgx = long_exponent(zx);
        lgy = long_exponent(zy);
      } else {
        lgx = long_exponent(bmx);
        lgy = long_exponent(bmy);
      }
      lmx = lm.x;
      lmy = lm.y;
    };


    // the strips, each run until both halves' bottoms are in the window
    bool fail_x = false, fail_y = !two;
    for (int strip = 0; strip < nstrips && (okx || oky); ++strip) {
      const bool last = strip == nstrips - 1;
      const int ns = min(SR, n - strip * SR);
      const int used = (ns + R - 1) / R;  // lanes holding read rows
      const int lrows = lane < used ? min(R, ns - lane * R) : 0;
      const int in0 = strip == 0 ? kLongStart : 0;  // exponent of the strip's input
      if (g > 0 && strip < prof_len) {
        // the first pair's decay of each lane, aiming its bottom at 2^0
        const int d = lane < used ? (int)prof[strip * kWarp + lane] : 0;
        klx = lane < used ? max(-96, min(120, d - (lane == 0 ? in0 : 0))) : 0;
        kly = klx;
      } else {
        // the predicted boost spread evenly over the lanes holding read rows
        klx = lane < used ? (lane + 1) * Bx / used - lane * Bx / used : 0;
        kly = lane < used ? (lane + 1) * By / used - lane * By / used : 0;
      }
      for (int attempt = 0;; ++attempt) {
        run_strip(strip, last);
        if (qv.strip_runs != nullptr && lane == 0) {
          atomicAdd(qv.strip_runs, 1ull);
          if (attempt == 0) atomicAdd(qv.strip_runs + 1, 1ull);
        }
        const bool gx = !okx || (lgx >= kLongFloor && lgx < kLongCeil && lanes_in_window(lmx, used));
        const bool gy = !oky || (lgy >= kLongFloor && lgy < kLongCeil && lanes_in_window(lmy, used));
        if (gx && gy) break;
        if (attempt + 1 == kLongTries) {
          if (!gx) { okx = false; fail_x = true; }
          if (!gy) { oky = false; fail_y = true; }
          break;
        }
        // a half that left the window takes each lane's measured decay
        if (!gx) klx = relane(klx, lmx, used, lrows, in0, lane);
        if (!gy) kly = relane(kly, lmy, used, lrows, in0, lane);
      }
      // the strip's boost per half: the sum of its lanes' shares
      Bx = klx;
      By = kly;
#pragma unroll
      for (int o = 16; o; o >>= 1) {
        Bx += __shfl_xor_sync(FULL, Bx, o);
        By += __shfl_xor_sync(FULL, By, o);
      }
      // a half whose read decayed by more than kLongMaxRate bits per row so far
      // (with 64 bits of slack and the first strip's 2^60 start) is beyond what
      // this tier keeps exact (alignment families that trade places across
      // rows sit far below the row maximum): it goes to the drift and FP64 tiers
      const int cap = kLongMaxRate * (Nrows + ns) + 64 + kLongStart;
      if (okx && Dx + Bx + in0 - lgx > cap) { okx = false; fail_x = true; }
      if (oky && Dy + By + in0 - lgy > cap) { oky = false; fail_y = true; }
      if (g == 0 && strip == prof_len && strip < kLongProfStrips && (okx || oky)) {
        const int lg = long_exponent(okx ? lmx : lmy);
        int in = __shfl_up_sync(FULL, lg, 1);
        if (lane == 0) in = in0;
        prof[strip * kWarp + lane] = (short)(lane < used ? (okx ? klx : kly) + in - lg : 0);
        ++prof_len;
      }
      // the boosts of the strip count into the exponent (plus the first strip's start)
      if (!last) {
        // the next strip reads this one's boundary brought to 2^0 (|lg| <= 60, so
        // one exact factor); its boost is the read's mean decay rate so far
        // times its rows
        const int ksx = okx ? -lgx : 0, ksy = oky ? -lgy : 0;
        inx = ksx;
        iny = ksy;
        const int ns1 = min(SR, n - (strip + 1) * SR);
        Nrows += ns;
        if (okx) {
          Ex += Bx + in0 + ksx;
          Dx += Bx + in0 - lgx;
          Bx = max(0, min(4 * ns1, Dx * ns1 / Nrows));
        }
        if (oky) {
          Ey += By + in0 + ksy;
          Dy += By + in0 - lgy;
          By = max(0, min(4 * ns1, Dy * ns1 / Nrows));
        }
      } else {
        Ex += Bx + in0;
        Ey += By + in0;
      }
    }

    // ln of the final sum z = f 2^e (f in [1/2, 1)) less the boosts: the bits
    // do not depend on which powers of two the boosts took
    if (lane == kWarp - 1) {
      const int64_t o1 = w.out_begin + g;
      if (okx && !fail_x) {
        int e;
        const double f = frexp(zx, &e);
        bv.out[o1] = log(f) - (sc.ln_c + log((double)(m1 + 1))) + lnN + (double)(e - Ex) * kLn2;
      } else {
        bv.out[o1] = __longlong_as_double(0x7ff8000000000000LL);
        spill_pair<float>(qv, w.read, h1, o1);
      }
      if (two) {
        if (oky && !fail_y) {
          int e;
          const double f = frexp(zy, &e);
          bv.out[o1 + 1] = log(f) - (sc.ln_c + log((double)(m2 + 1))) + lnN + (double)(e - Ey) * kLn2;
        } else {
          bv.out[o1 + 1] = __longlong_as_double(0x7ff8000000000000LL);
          spill_pair<float>(qv, w.read, h2, o1 + 1);
        }
      }
    }
    __syncwarp();
  }
}

// Persistent kernel of the long-read items (FP32 semiglobal primary tier):
// every warp pulls items from qv.head (or walks them in the fixed round-robin
// order of the plain schedule).  Items whose read has another rows-per-lane
// count than R are not in its list.
template <int R, int kBlocks>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp, kBlocks)
pairhmm_long_kernel(const BatchView bv, const QueueView qv, const Tables<float>* __restrict__ gtab,
                    const Scalars<float> sc) {
  __shared__ Tables<float> tab;
  __shared__ float4 rings[kWarpsPerBlock][2][kWarp];
  __shared__ short profs[kWarpsPerBlock][kLongProfStrips * kWarp];
  {
    const int words = (int)(sizeof(Tables<float>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(gtab);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1);
  const long long gw = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  float4* scratch = reinterpret_cast<float4*>(qv.scratch) + gw * qv.scratch_stride;
  const long long stride = (long long)gridDim.x * kWarpsPerBlock;
  long long next = gw;
  for (;;) {
    unsigned long long i = 0;
    if (qv.static_order) {
      i = (unsigned long long)next;
      next += stride;
    } else {
      if (lane == 0) i = atomicAdd(qv.head, 1ull);
      i = __shfl_sync(0xffffffffu, i, 0);
    }
    if ((long long)i >= qv.n_items) break;
    process_long<R>(bv, qv, qv.items[i], &tab, sc, lane, scratch, rings[threadIdx.x >> 5][0],
                    rings[threadIdx.x >> 5][1], profs[threadIdx.x >> 5]);
  }
}

// ---- block per pair: the warps of a CTA split each strip -----------------------
//
// The CTA's kWarpsPerBlock warps run one item together over tall strips of
// W = kWarpsPerBlock times 32 R rows: warp w owns rows 32 R w .. 32 R (w+1) - 1
// of each tall strip, so a pair's strips run side by side instead of one after
// another, which shortens a long pair's latency W-fold when few long pairs
// fill the GPU.  Warp w's bottom row reaches warp w+1 through a shared-memory
// ring: warp w runs kLongLag steps behind warp w-1 and the block meets at a
// barrier every kLongChunk steps, so a column is always written one chunk or
// more before it is read and overwritten two chunks or more after (lane 31 of
// warp w-1 produces column c at its step c + 31, lane 0 of warp w reads it at
// its step c, kLongLag - 31 > kLongChunk steps later; the ring holds
// kLongRing >= kLongChunk + kLongLag columns).  Every warp takes the same
// number of chunks and barriers whatever its share of the strip, so the
// barriers always complete.  Each warp has its own boost rate (the decay of
// its own rows, measured at its bottom), the tall strip's boundary is brought
// to 2^0 exactly as the next tall strip loads it, and a tall strip whose warps' bottoms leave the window
// is run again with each warp's rate corrected by what it measured.
constexpr int kLongChunk = 32;
constexpr int kLongLag = 64;
constexpr int kLongRing = 128;
static_assert(kLongLag - (kWarp - 1) > kLongChunk, "a column must be written a chunk before it is read");
static_assert(kLongRing >= kLongChunk + kLongLag, "the ring must hold every column in flight");

struct LongBlockShared {
  float4 hand[kWarpsPerBlock - 1][kLongRing];  // warp w -> w+1 bottom rows (s.x, u.x, s.y, u.y)
  float4 ring0[kWarp];                          // warp 0: boundary records of the tall strip above
  int lg[kWarpsPerBlock][2];                    // bottom exponents of the last run
  int B[kWarpsPerBlock][2];                     // boost bits of each warp's rows
  int D[2];                                     // decay (bits) over the rows done so far
  int rows;                                     // those rows
  double z[2];                                  // final sums
  long long item;
};

template <int R>
__device__ __noinline__ void process_long_block(const BatchView bv, const QueueView qv, const WorkItem w,
                                                const Tables<float>* __restrict__ tb, const Scalars<float> sc,
                                                const int lane, const int wid, float4* __restrict__ scratch,
                                                LongBlockShared& sh) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr double kLn2 = 0.6931471805599453094;
  constexpr int SR = kWarp * R;
  constexpr int NW = kWarpsPerBlock;
  constexpr int H = NW * SR;
  const int tid = wid * kWarp + lane;
  const int64_t roff = bv.read_off[w.read];
  const int n = (int)(bv.read_off[w.read + 1] - roff);
  const uint8_t* __restrict__ rbase = bv.read_bases + roff;
  const uint8_t* __restrict__ rqual = bv.read_quals + roff;
  const bool two = w.nhap > 1;
  const int64_t h1 = w.hap_begin, h2 = two ? w.hap_begin + 1 : w.hap_begin;
  const int64_t ho1 = bv.hap_off[h1], ho2 = bv.hap_off[h2];
  const int m1 = (int)(bv.hap_off[h1 + 1] - ho1), m2 = (int)(bv.hap_off[h2 + 1] - ho2);
  const uint8_t* __restrict__ hp1 = bv.hap_bases + ho1 - 1;
  const uint8_t* __restrict__ hp2 = bv.hap_bases + ho2 - 1;
  const int M = max(m1, m2);
  const int ntall = (n + H - 1) / H;
  const long long half = qv.scratch_stride / 2;
  const int steps = M + 1 + (kWarp - 1);
  const int chunks = (steps + (NW - 1) * kLongLag + kLongChunk - 1) / kLongChunk;

  double lnN = 0.0;
  for (int i = lane; i < n; i += kWarp) lnN += tb->lnN[rqual[i]];
#pragma unroll
  for (int o = 16; o; o >>= 1) lnN += __shfl_xor_sync(FULL, lnN, o);
  const float A = tb->A[rqual[n - 1]];
  const float2 k2 = make_float2(sc.k2, sc.k2), x = make_float2(sc.x, sc.x);
  const float cin = sc.c * pow2T(kLongStart, 0.f);

  if (tid < NW * 2) sh.B[tid >> 1][tid & 1] = 0;
  if (tid < 2) sh.D[tid] = 0;
  if (tid == 0) sh.rows = 0;
  __syncthreads();
  // per half, identical in every thread: total exponent, still in play
  int Ex = 0, Ey = 0;
  bool okx = true, oky = two;
  int inx = 0, iny = 0;  // shifts that bring the boundary above to 2^0, per half

  // one run of tall strip S; the warps' bottom exponents (or the final sums) land in sh
  auto run_tall = [&](const int S, const int active, const bool last) {
    const int i0 = S * H + wid * SR;                 // first row of this warp
    const int ns = min(SR, n - i0);                  // its read rows (<= 0: idle)
    const int lanes_used = ns > 0 ? (ns + R - 1) / R : 0;
    const int Bx = sh.B[wid][0], By = sh.B[wid][1];
    LongRows<R> rw;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = i0 + lane * R + r;
      if (i < n) {
        const unsigned q = rqual[i];
        rw.rb[r] = rbase[i];
        rw.miss[r] = tb->miss[q];
        const float K = tb->K[q], X = (i == n - 1) ? A : tb->X[q];
        rw.K[r] = make_float2(K, K);
        rw.X[r] = make_float2(X, X);
      } else {
        rw.rb[r] = kNeverBase;
        rw.miss[r] = 0.f;
        rw.K[r] = make_float2(0.f, 0.f);
        rw.X[r] = make_float2(1.f, 1.f);
      }
      rw.W[r] = make_float2(0.f, 0.f);
      rw.s[r] = make_float2(0.f, 0.f);
    }
    int kx = 0, ky = 0;
    if (lane < lanes_used) {
      kx = (lane + 1) * Bx / lanes_used - lane * Bx / lanes_used;
      ky = (lane + 1) * By / lanes_used - lane * By / lanes_used;
    }
    boost_row0(rw, make_float2(pow2T(kx, 0.f), pow2T(ky, 0.f)));
    float4* const src = scratch + (long long)(S & 1) * half;
    float4* const dst = scratch + (long long)((S + 1) & 1) * half;
    // the tall strip above's boundary, brought to 2^0 as warp 0 loads it
    const float fsx = pow2T(inx, 0.f), fsy = pow2T(iny, 0.f);
    const bool bottom = wid == active - 1;  // this warp's bottom row is the tall strip's
    float2 s_top = make_float2(0.f, 0.f), u_bot = make_float2(0.f, 0.f), acc32 = make_float2(0.f, 0.f);
    double accx = 0.0, accy = 0.0;
    float bmx = 0.f, bmy = 0.f;
    float4 nxt = make_float4(0.f, 0.f, 0.f, 0.f);
    auto load_window = [&](int base) -> float4 {
      const int p = base + lane;
      if (S == 0 || p > M) return make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 v = src[p];
      return make_float4(v.x * fsx, v.y * fsx, v.z * fsy, v.w * fsy);
    };
    if (wid == 0) nxt = load_window(0);
    for (int k = 0; k < chunks; ++k) {
      for (int uu = 0; uu < kLongChunk; ++uu) {
        const int t = k * kLongChunk + uu - wid * kLongLag;  // this warp's step (warp-uniform)
        if (wid >= active || t < 0 || t >= steps) continue;
        if (wid == 0 && (t & (kWarp - 1)) == 0) {
          __syncwarp();
          sh.ring0[lane] = nxt;
          __syncwarp();
          nxt = load_window(t + kWarp);
        }
        const int p = t - lane;
        float2 u_in = shfl_up2(u_bot);
        float2 s_in = shfl_up2(rw.s[R - 1]);
        if (lane == 0) {
          if (wid > 0) {
            const float4 rec = sh.hand[wid - 1][t & (kLongRing - 1)];
            s_in = make_float2(rec.x, rec.z);
            u_in = make_float2(rec.y, rec.w);
          } else if (S == 0) {
            u_in = make_float2(cin, cin);
            s_in = u_in;
          } else {
            const float4 rec = sh.ring0[t & (kWarp - 1)];
            s_in = make_float2(rec.x, rec.z);
            u_in = make_float2(rec.y, rec.w);
          }
        }
        const bool inside = p >= 0 && p <= M;
        const uint32_t hbx = (inside && p > 0) ? (uint32_t)hp1[min(p, m1)] : kNeverBase;
        const uint32_t hby = (inside && p > 0) ? (uint32_t)hp2[min(p, m2)] : kNeverBase;
        column_long<R>(rw, hbx, hby, p > 0 ? s_top : make_float2(0.f, 0.f), u_in, k2, x, u_bot);
        if (p <= 0) {
#pragma unroll
          for (int r = 0; r < R; ++r) rw.W[r] = make_float2(0.f, 0.f);
        }
        s_top = s_in;
        if (lane == kWarp - 1 && inside) {
          const float4 rec = make_float4(rw.s[R - 1].x, u_bot.x, rw.s[R - 1].y, u_bot.y);
          if (bottom && last) {
            if (p <= m1) acc32.x += u_bot.x;
            if (p <= m2) acc32.y += u_bot.y;
            if ((p & 7) == 7) {
              accx += (double)acc32.x;
              accy += (double)acc32.y;
              acc32 = make_float2(0.f, 0.f);
            }
          } else {
            if (bottom) dst[p] = rec;
            else sh.hand[wid][p & (kLongRing - 1)] = rec;
            if (p <= m1) bmx = fmaxf(bmx, fmaxf(rec.x, rec.y));
            if (p <= m2) bmy = fmaxf(bmy, fmaxf(rec.z, rec.w));
          }
        }
      }
      __syncthreads();
    }
    if (wid < active) {
      if (bottom && last) {
        const double zx = __shfl_sync(FULL, accx + (double)acc32.x, kWarp - 1);
        const double zy = __shfl_sync(FULL, accy + (double)acc32.y, kWarp - 1);
        if (lane == 0) {
          sh.z[0] = zx;
          sh.z[1] = zy;
          sh.lg[wid][0] = long_exponent(zx);
          sh.lg[wid][1] = long_exponent(zy);
        }
      } else {
        const float bx = __shfl_sync(FULL, bmx, kWarp - 1), by = __shfl_sync(FULL, bmy, kWarp - 1);
        if (lane == 0) {
          sh.lg[wid][0] = long_exponent(bx);
          sh.lg[wid][1] = long_exponent(by);
        }
      }
    }
    __syncthreads();
  };

  bool fail_x = false, fail_y = !two;
  for (int S = 0; S < ntall && (okx || oky); ++S) {
    const int rows = min(H, n - S * H);
    const int active = (rows + SR - 1) / SR;
    const bool last = S == ntall - 1;
    const int start = S == 0 ? kLongStart : 0;
    auto rows_of = [&](int wi) { return min(SR, rows - wi * SR); };
    for (int attempt = 0;; ++attempt) {
      run_tall(S, active, last);
      // every thread reads the same exponents and takes the same decisions
      bool gx = !okx, gy = !oky;
      if (!gx) {
        gx = true;
        for (int wi = 0; wi < active; ++wi) gx &= sh.lg[wi][0] >= kLongFloor && sh.lg[wi][0] < kLongCeil;
      }
      if (!gy) {
        gy = true;
        for (int wi = 0; wi < active; ++wi) gy &= sh.lg[wi][1] >= kLongFloor && sh.lg[wi][1] < kLongCeil;
      }
      if (gx && gy) break;
      if (attempt + 1 == kLongTries) {
        if (!gx) { okx = false; fail_x = true; }
        if (!gy) { oky = false; fail_y = true; }
        break;
      }
      // each warp's rows get their own measured decay (in: the warp above's
      // bottom, or the tall strip's input), aiming every bottom at 2^0.  A
      // warp whose bottom over- or underflowed, or whose input did, takes the
      // decay rate (bits per row) measured by the lowest warp above it that
      // could measure one, so a first tall strip converges in two or three
      // runs rather than one warp per run
      __syncthreads();
      if (tid == 0) {
        for (int hf = 0; hf < 2; ++hf) {
          if (hf == 0 ? gx : gy) continue;
          int rate_num = -1, rate_den = 1;  // last measured decay and its rows
          bool input_ok = true;
          for (int wi = 0; wi < active; ++wi) {
            const int in = wi == 0 ? start : sh.lg[wi - 1][hf];
            const int lg = sh.lg[wi][hf];
            const int ns = rows_of(wi);
            int B = sh.B[wi][hf];
            input_ok = input_ok && in != 1024 && in != -1024;
            if (input_ok && lg != 1024 && lg != -1024) {
              const int d = B + in - lg;  // this warp's own decay
              rate_num = d;
              rate_den = ns;
              B = d - (wi == 0 ? start : 0);
            } else if (rate_num >= 0) {
              B = rate_num * ns / rate_den - (wi == 0 ? start : 0);
            } else if (input_ok) {
              B += lg == 1024 ? -ns / 2 : ns / 2;
            }
            sh.B[wi][hf] = max(-4 * ns, min(4 * ns, B));
          }
        }
      }
      __syncthreads();
    }
    // exponent bookkeeping, the shift of the boundary and the rates
    // of the next tall strip (each warp's decay, scaled to its next rows)
    const int lgb_x = sh.lg[active - 1][0], lgb_y = sh.lg[active - 1][1];
    int sumBx = 0, sumBy = 0;
    for (int wi = 0; wi < active; ++wi) { sumBx += sh.B[wi][0]; sumBy += sh.B[wi][1]; }
    if (!last) {
      const int ksx = okx ? -lgb_x : 0, ksy = oky ? -lgb_y : 0;
      inx = ksx;
      iny = ksy;
      if (okx) Ex += sumBx + start + ksx;
      if (oky) Ey += sumBy + start + ksy;
      const int rows1 = min(H, n - (S + 1) * H);
      __syncthreads();
      if (tid == 0) {
        // every warp of the next tall strip takes the read's mean decay rate
        // so far (the decays of this tall strip's warps telescope to its
        // boosts plus its input minus its bottom), times its rows
        sh.rows += rows;
        for (int hf = 0; hf < 2; ++hf) {
          sh.D[hf] += (hf == 0 ? sumBx : sumBy) + start - sh.lg[active - 1][hf];
          for (int wi = 0; wi < NW; ++wi) {
            const int ns1 = max(0, min(SR, rows1 - wi * SR));
            sh.B[wi][hf] = max(0, min(4 * ns1, (int)((long long)sh.D[hf] * ns1 / sh.rows)));
          }
        }
      }
      __syncthreads();
    } else {
      if (okx) Ex += sumBx + start;
      if (oky) Ey += sumBy + start;
    }
  }

  if (tid == 0) {
    const double lnC1 = sc.ln_c + log((double)(m1 + 1));
    const double lnC2 = sc.ln_c + log((double)(m2 + 1));
    if (okx && !fail_x) {
      bv.out[w.out_begin] = log(sh.z[0]) - lnC1 + lnN - (double)Ex * kLn2;
    } else {
      bv.out[w.out_begin] = __longlong_as_double(0x7ff8000000000000LL);
      spill_pair<float>(qv, w.read, h1, w.out_begin);
    }
    if (two) {
      if (oky && !fail_y) {
        bv.out[w.out_begin + 1] = log(sh.z[1]) - lnC2 + lnN - (double)Ey * kLn2;
      } else {
        bv.out[w.out_begin + 1] = __longlong_as_double(0x7ff8000000000000LL);
        spill_pair<float>(qv, w.read, h2, w.out_begin + 1);
      }
    }
  }
  __syncthreads();
}

// Persistent block-per-pair kernel of the long-read items: the whole CTA takes
// one item at a time (thread 0 pulls it, a barrier hands it to the block).
// Each CTA uses the strip scratch slot of its first warp.
template <int R, int kBlocks>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp, kBlocks)
pairhmm_long_block_kernel(const BatchView bv, const QueueView qv, const Tables<float>* __restrict__ gtab,
                          const Scalars<float> sc) {
  __shared__ Tables<float> tab;
  __shared__ LongBlockShared sh;
  {
    const int words = (int)(sizeof(Tables<float>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(gtab);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  const int lane = threadIdx.x & (kWarp - 1);
  const int wid = threadIdx.x >> 5;
  float4* scratch = reinterpret_cast<float4*>(qv.scratch) + (long long)blockIdx.x * kWarpsPerBlock * qv.scratch_stride;
  long long next = blockIdx.x;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      if (qv.static_order) {
        sh.item = next;
        next += gridDim.x;
      } else {
        sh.item = (long long)atomicAdd(qv.head, 1ull);
      }
    }
    __syncthreads();
    const long long i = sh.item;
    if (i >= qv.n_items) break;
    process_long_block<R>(bv, qv, qv.items[i], &tab, sc, lane, wid, scratch, sh);
  }
}

}  // namespace vd
