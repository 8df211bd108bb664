// Device code of the PairHMM wavefront.  Included once per (type, mode)
// instantiation unit; see pairhmm_core.cuh for the model and the scaling.
#pragma once
#include <climits>
#include <cmath>
#include <type_traits>
#include "pairhmm_core.cuh"

namespace vd {

template <typename T> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

__device__ __forceinline__ float fmaT(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmaT(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float maxT(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double maxT(double a, double b) { return fmax(a, b); }

// v *= f when the read base a differs from the haplotype base b: one compare
// and one predicated multiply (a match leaves v untouched).
__device__ __forceinline__ void mul_if_ne(float& v, uint32_t a, uint32_t b, float f) {
  asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, %2;\n\t@p mul.rn.f32 %0, %0, %3;\n\t}"
      : "+f"(v) : "r"(a), "r"(b), "f"(f));
}
__device__ __forceinline__ void mul_if_ne(double& v, uint32_t a, uint32_t b, double f) {
  asm("{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, %2;\n\t@p mul.rn.f64 %0, %0, %3;\n\t}"
      : "+d"(v) : "r"(a), "r"(b), "d"(f));
}

// 2^k for k inside the normal range of T.
__device__ __forceinline__ float pow2T(int k, float) { return __int_as_float((k + 127) << 23); }
__device__ __forceinline__ double pow2T(int k, double) {
  return __longlong_as_double((long long)(k + 1023) << 52);
}

// The R rows a lane owns: per-row constants and the state of the column the
// lane finished last.
template <typename T, int R, bool GEN>
struct LaneRows {
  uint32_t rb[R];          // read base (0 for padding rows: never equals a base)
  T miss[R];               // mismatch factor
  T hit[GEN ? R : 1];      // match factor (only when some row has P0 > P1)
  T K[R], X[R];            // k1 f_i and (x/4) f_i
  T mu[R], om[R], s[R];    // mu, omega and s of the previous column
};

// One DP column of this lane.  s_top is s of the row above at column j-1,
// u_top is u of the row above at column j.  With TAP the bottom row's mu, nu
// and omega are returned for the anchored end cell.
template <typename T, int R, bool GEN, bool TAP>
__device__ __forceinline__ void column(LaneRows<T, R, GEN>& w, uint32_t hb, T s_top, T u_top,
                                       T k2, T x, T& u_bot, T& tap_mu, T& tap_nu, T& tap_om) {
  T s_above = s_top;
  T nu = u_top;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    T mu_new = s_above;
    if (GEN) {
      mu_new = s_above * (w.rb[r] == hb ? w.hit[r] : w.miss[r]);
    } else {
      mul_if_ne(mu_new, w.rb[r], hb, w.miss[r]);
    }
    const T om_new = fmaT(x, w.om[r], w.mu[r]);
    const T u_new = fmaT(w.X[r], nu, mu_new);
    const T s_new = fmaT(k2, om_new, fmaT(w.K[r], nu, mu_new));
    if (TAP && r == R - 1) { tap_mu = mu_new; tap_nu = nu; tap_om = om_new; }
    s_above = w.s[r];
    w.mu[r] = mu_new;
    w.om[r] = om_new;
    w.s[r] = s_new;
    nu = u_new;
  }
  u_bot = nu;
}

struct ItemRef {
  WorkItem w;
  bool use_sel;   // resolve haplotypes / outputs through hap_sel / out_sel
  int tier;
};

template <typename T>
__device__ __forceinline__ void spill_pair(const QueueView& qv, int32_t read, int64_t hap, int64_t out) {
  if (qv.spill == nullptr) return;
  const unsigned long long slot = atomicAdd(qv.spill_count, 1ull);
  if ((long long)slot < qv.spill_cap) {
    qv.spill[slot] = RescueEntry{read, (int32_t)hap, out};
  } else {
    atomicExch(qv.error_flag, 1);
  }
}

constexpr int kUnroll = 8;

// The drift tier (FP32, semiglobal) rescores the pairs the primary tier
// spilled.  Error-rich long reads lose more per strip
// than the FP32 range holds (8% errors at reported Q30: about 1 bit per row),
// so each row's constants are multiplied by an exact power of two 2^k_i that
// cancels the decay: Bs bits per strip, spread over its rows.  Bs is measured
// as the read goes (the next strip takes the decay left over at the bottom of
// this one) and a strip whose bottom leaves the window [2^-60, 2^60) is run
// again with Bs corrected by the measured exponent (its input boundary is kept
// in the other half of the warp's scratch).  A read of one strip spilled
// because its likelihood lies below the primary tier's range; its lanes each
// take their own boost, measured lane by lane (a variant or a cluster of
// errors concentrates the decay in a few rows).  What still fails goes to FP64.
constexpr int kDriftTries = 6;

// Row layout of one read (lane L, register r of strip s holds row
// i = s*32R + L*R + r - v, 0-based):
//  * semiglobal (v = 0): rows below the read pass the last row's u down the
//    column (miss = 0, K = 0, X = 1), and the last row's X is alpha*f_n, so
//    lane 31's bottom u is the scaled (M + I)[n][j] the result sums;
//  * anchored: the read ends at lane 31's bottom register of the last strip and
//    v >= 1 virtual rows sit on top: "zero rows" (miss = K = X = 0) and, just
//    above row 1, an emulator of row 0 (miss = 1, K = X = 0) that is fed
//    s(-1) = c at each column 0; its omega recurrence regenerates the anchored
//    row-0 deletions D[0][j] = g x^(j-1) (anchored.cpp:9).
constexpr uint32_t kNeverBase = 0x10000u;  // compares unequal to every base byte

template <typename T, int R, bool GEN, bool ANCH, bool DRIFT = false>
__device__ __noinline__ void process_item(const BatchView bv, const QueueView qv, const ItemRef it,
                                          const Tables<T>* __restrict__ tb, const Scalars<T> sc,
                                          const int lane, typename Vec2<T>::type* __restrict__ scratch) {
  using T2 = typename Vec2<T>::type;
  constexpr unsigned FULL = 0xffffffffu;
  constexpr double kLn2 = 0.6931471805599453094;
  const WorkItem& w = it.w;
  const int64_t roff = bv.read_off[w.read];
  const int n = (int)(bv.read_off[w.read + 1] - roff);
  const uint8_t* __restrict__ rbase = bv.read_bases + roff;
  const uint8_t* __restrict__ rqual = bv.read_quals + roff;
  const int K = w.nhap;
  constexpr int SR = kWarp * R;
  const int n_rows = n + (ANCH ? 1 : 0);
  const int nstrips = (n_rows + SR - 1) / SR;
  const int v = ANCH ? nstrips * SR - n : 0;

  auto hap_index = [&](int k) -> int64_t {
    return it.use_sel ? (int64_t)bv.hap_sel[w.hap_begin + k] : w.hap_begin + k;
  };
  auto out_index = [&](int k) -> int64_t {
    return it.use_sel ? bv.out_sel[w.out_begin + k] : w.out_begin + k;
  };

  // sum_i ln N_i over the read (FP64), identical on every lane
  double lnN = 0.0;
  for (int i = lane; i < n; i += kWarp) lnN += tb->lnN[rqual[i]];
#pragma unroll
  for (int o = 16; o; o >>= 1) lnN += __shfl_xor_sync(FULL, lnN, o);

  const T A = tb->A[rqual[n - 1]];
  const T k2 = sc.k2, x = sc.x, c0 = sc.c, gfin = sc.gfin;
  int E = 0;          // total power-of-two scaling: strip renormalisations (and the drift tier's row boosts)
  bool fail = false;  // a strip boundary left the range

  // drift tier: per-row power-of-two boosts, strips re-run when they leave the
  // window; the scratch holds two boundaries (read one, write the other)
  constexpr bool kCanDrift = DRIFT && std::is_same<T, float>::value && GEN && !ANCH;
  constexpr bool drift = kCanDrift;
  const long long half = drift ? qv.scratch_stride / 2 : qv.scratch_stride;
  int strip_lg = 0;     // drift: exponent of the strip's bottom maximum (or +-1024: inf / zero)
  double zkeep = 0.0;   // drift: the last strip's final sum, on lane 31
  // drift, reads of one strip: each lane's own boost bits (spread over its read
  // rows) and the maximum of its bottom row's u over the columns of the last run
  bool lane_boost = false;
  int kl_lane = 0;
  T lmax_keep = T(0);

  // One strip of rows (Bs: the drift tier's boost bits for the strip, else 0).
  // FIRST and LAST are compile-time tags, so the steady loop carries no
  // per-step test of the strip position.  Returns false when the strip's
  // bottom boundary left [strip_floor, strip_ceil).
  auto run_strip = [&](auto first_tag, auto last_tag, const int strip, const int Bs) -> bool {
    constexpr bool FIRST = decltype(first_tag)::value;
    constexpr bool last = decltype(last_tag)::value;
    const bool lane0 = lane == 0;
    LaneRows<T, R, GEN> rw;
    const int row0 = strip * SR + lane * R - v;
    // the boundary this strip reads and the one it writes
    T2* const src = scratch + (drift ? (long long)(strip & 1) * half : 0ll);
    T2* const dst = scratch + (drift ? (long long)((strip + 1) & 1) * half : 0ll);
    const int ns = min(SR, n - strip * SR);  // read rows of the strip (drift: semiglobal, v = 0)
    int emu = -1;  // register of the anchored row-0 emulator in this lane
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = row0 + r;
      if (i >= 0 && i < n) {
        const unsigned q = rqual[i];
        rw.rb[r] = rbase[i];
        rw.miss[r] = tb->miss[q];
        if (GEN) rw.hit[r] = tb->hit[q];
        rw.K[r] = tb->K[q];
        rw.X[r] = (!ANCH && i == n - 1) ? A : tb->X[q];
        if constexpr (kCanDrift) {
          {
            // row il of the strip gets k = floor((il+1) Bs / ns) - floor(il Bs / ns),
            // or its share of the lane's own boost (the lane's read rows split it)
            const int il = i - strip * SR;
            const int lrows = min(R, n - lane * R);
            const int kr = lane_boost ? (r + 1) * kl_lane / lrows - r * kl_lane / lrows
                                      : (il + 1) * Bs / ns - il * Bs / ns;
            const T f = pow2T(kr, T(0));
            rw.miss[r] *= f;
            rw.hit[r] *= f;
            rw.K[r] *= f;
            rw.X[r] *= f;
          }
        }
      } else {
        const bool emulator = ANCH && i == -1;
        if (emulator) emu = r;
        rw.rb[r] = kNeverBase;
        rw.miss[r] = emulator ? T(1) : T(0);
        if (GEN) rw.hit[r] = rw.miss[r];
        rw.K[r] = T(0);
        rw.X[r] = (!ANCH && i >= n) ? T(1) : T(0);
      }
      rw.mu[r] = T(0);
      rw.om[r] = T(0);
      rw.s[r] = T(0);
    }

    int kL = -1;            // haplotype this lane is in
    int next_reset = 0;     // stream position of this lane's next column 0
    int S_cur = -1;         // stream position of this lane's current column 0
    const uint8_t* hp = bv.hap_bases;  // hp[p] = haplotype base at stream position p
    T s_top = T(0), u_bot = T(0);
    T acc32 = T(0), cap = T(0), rmax = T(0), bmax = T(0);
    T lmax = T(0);  // drift: maximum of this lane's bottom-row u
    double acc64 = 0.0;

    auto finalize = [&](int k) {
      const int64_t h = hap_index(k);
      const int64_t o = out_index(k);
      const int m = (int)(bv.hap_off[h + 1] - bv.hap_off[h]);
      const double Zs = ANCH ? (double)cap : acc64 + (double)acc32;
      // anchored.cpp:24 returns ln(max(1e-300, Z / S_n)) + ln S_n, S_n the max of
      // (M+I+D) over the last row: the clamp binds when the end cell lies more
      // than 1e-300 below that row maximum
      const double Zc = ANCH ? fmax(Zs, 1e-300 * (double)rmax) : Zs;
      const double lnC0 = sc.ln_c + (ANCH ? 0.0 : log((double)(m + 1)));
      if constexpr (drift) {
        zkeep = Zs;  // checked (and written) once the strip is done
        return;
      }
      const bool ok = !fail && Zs >= (double)sc.final_floor && Zs < HUGE_VAL;
      if (ok || qv.spill == nullptr) {
        bv.out[o] = (Zc > 0.0 ? log(Zc) : -HUGE_VAL) - lnC0 + lnN - (double)E * kLn2;
      } else {
        bv.out[o] = __longlong_as_double(0x7ff8000000000000LL);
        spill_pair<T>(qv, w.read, h, o);
      }
    };

    auto zero_state = [&]() {
#pragma unroll
      for (int r = 0; r < R; ++r) { rw.mu[r] = T(0); rw.om[r] = T(0); rw.s[r] = T(0); }
      s_top = T(0);
      acc32 = T(0);
      acc64 = 0.0;
      cap = T(0);
      rmax = T(0);
      if (ANCH && FIRST) {
        // the emulator row reads s(-1) = c from the row above at column 0
        if (emu == 0) s_top = c0;
#pragma unroll
        for (int r = 1; r < R; ++r)
          if (emu == r) rw.s[r - 1] = c0;
      }
    };

    // the final-row tap (lane 31): semiglobal sums (M + I)[n][j] over every
    // column -- it arrives as the bottom u -- and anchored keeps (M + I + D) of
    // the latest column and the running row maximum
    auto accumulate = [&](T tmu, T tnu, T tom) {
      if (ANCH) {
        cap = fmaT(gfin, tom, fmaT(A, tnu, tmu));
        rmax = maxT(rmax, cap);
      } else {
        acc32 += u_bot;
      }
    };

    // Boundary records of the strip above, for lane 0 (whose stream position is
    // the step index t): each lane loads one record of the next 32 positions in
    // one coalesced access, a window ahead of use, and a shuffle hands lane 0
    // its record, so no step waits on memory.  A position is read here before
    // lane 31 overwrites it with this strip's own boundary (31 or more steps
    // later, past a __syncwarp).
    T2 pf_cur = {T(0), T(0)}, pf_nxt = {T(0), T(0)};
    auto pf_load = [&](int base) -> T2 {
      const long long q = (long long)base + lane;
      return q < half ? src[q] : T2{T(0), T(0)};
    };
    if (!FIRST) {
      pf_cur = pf_load(0);
      pf_nxt = pf_load(kWarp);
    }
    auto boundary = [&](int t) -> T2 {
      const int k = t & (kWarp - 1);
      if (k == 0 && t > 0) {
        pf_cur = pf_nxt;
        pf_nxt = pf_load(t + kWarp);
      }
      T2 r;
      r.x = __shfl_sync(FULL, pf_cur.x, k);
      r.y = __shfl_sync(FULL, pf_cur.y, k);
      return r;
    };

    // step with per-lane haplotype bookkeeping (ramps and short haplotypes)
    auto gstep = [&](int t) {
      const int p = t - lane;
      T u_in = __shfl_up_sync(FULL, u_bot, 1);
      T s_in = __shfl_up_sync(FULL, rw.s[R - 1], 1);
      if (p == next_reset) {
        if (last && kL >= 0 && lane == kWarp - 1) finalize(kL);
        ++kL;
        zero_state();
        S_cur = p;
        if (kL < K) {
          const int64_t h = hap_index(kL);
          const int64_t ho = bv.hap_off[h];
          const int m = (int)(bv.hap_off[h + 1] - ho);
          hp = bv.hap_bases + ho - 1 - p;
          next_reset = p + m + 1;
        } else {
          next_reset = INT_MAX;
        }
      }
      const bool active = kL >= 0 && kL < K;
      const bool col0 = p == S_cur;
      const uint32_t hb = (active && !col0) ? (uint32_t)hp[p] : 0u;
      T iu, is;
      if (FIRST) {
        iu = ANCH ? T(0) : c0;
        is = iu;
      } else {
        T2 rec = boundary(t);
        if (!active) rec = T2{T(0), T(0)};
        iu = rec.y;
        is = rec.x;
      }
      u_in = lane0 ? iu : u_in;
      s_in = lane0 ? is : s_in;
      T tmu = T(0), tnu = T(0), tom = T(0);
      column<T, R, GEN, ANCH>(rw, hb, s_top, u_in, k2, x, u_bot, tmu, tnu, tom);
      if constexpr (drift) {
        if (active) lmax = maxT(lmax, u_bot);
      }
      s_top = s_in;
      if (last) {
        accumulate(tmu, tnu, tom);
        // lane 31 moves its row sum into FP64 after its columns 8r+7 (by
        // column, as the two-read path does, so both give the same bits)
        if (!ANCH && lane == kWarp - 1 && ((p - S_cur) & 7) == 7) { acc64 += (double)acc32; acc32 = T(0); }
      } else {
        if (lane == kWarp - 1 && active) {
          dst[p] = T2{rw.s[R - 1], u_bot};
          bmax = maxT(bmax, maxT(rw.s[R - 1], u_bot));
        }
        __syncwarp();
      }
    };

    // step with every lane inside the same haplotype at a column >= 1
    auto sstep = [&](uint32_t hb, int p, int t) {
      T u_in = __shfl_up_sync(FULL, u_bot, 1);
      T s_in = __shfl_up_sync(FULL, rw.s[R - 1], 1);
      T iu, is;
      if (FIRST) {
        iu = ANCH ? T(0) : c0;
        is = iu;
      } else {
        const T2 rec = boundary(t);
        iu = rec.y;
        is = rec.x;
      }
      u_in = lane0 ? iu : u_in;
      s_in = lane0 ? is : s_in;
      T tmu = T(0), tnu = T(0), tom = T(0);
      column<T, R, GEN, ANCH>(rw, hb, s_top, u_in, k2, x, u_bot, tmu, tnu, tom);
      if constexpr (drift) lmax = maxT(lmax, u_bot);
      s_top = s_in;
      if (last) {
        accumulate(tmu, tnu, tom);
      } else if (lane == kWarp - 1) {
        dst[p] = T2{rw.s[R - 1], u_bot};
        bmax = maxT(bmax, maxT(rw.s[R - 1], u_bot));
      }
    };

    int t = 0;
    int S = 0;
    for (int k = 0; k <= K; ++k) {
      int mk = 0;
      if (k < K) {
        const int64_t h = hap_index(k);
        mk = (int)(bv.hap_off[h + 1] - bv.hap_off[h]);
      }
      const int Snext = S + mk + 1;
      const int gen_end = (k < K) ? min(S + kWarp, Snext) : S + kWarp;
      for (; t < gen_end; ++t) gstep(t);
      if (k < K) {
        // all lanes are inside haplotype k for t in [S + 32, Snext).  Lane
        // 31's column at step t is t - 31 - S; single steps bring it to a
        // multiple of 8, so every block of 8 ends on a column 8r+7
        const int lead = -(kWarp - 1) - S;
        for (; t < Snext && ((lead + t) & 7) != 0; ++t) {
          sstep((uint32_t)hp[t - lane], t - lane, t);
          if (last && !ANCH && ((lead + t) & 7) == 7) { acc64 += (double)acc32; acc32 = T(0); }
        }
        static_assert(kUnroll == 8, "blocks of 8 steps flush once, at their last column");
        for (; t + kUnroll <= Snext; t += kUnroll) {
          const uint8_t* q = hp + (t - lane);
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) sstep((uint32_t)q[u], t - lane + u, t + u);
          if (last && !ANCH) { acc64 += (double)acc32; acc32 = T(0); }
          if (!last) __syncwarp();
        }
        for (; t < Snext; ++t) sstep((uint32_t)hp[t - lane], t - lane, t);  // columns 8r..8r+6: no flush
      }
      S = Snext;
    }
    if constexpr (drift) lmax_keep = lmax;

    if (!last) {
      // renormalise the boundary the next strip starts from: its maximum is
      // brought to 2^target by an exact power of two, applied as two factors
      // so that any exponent shift stays representable
      __syncwarp();
      const T bm = __shfl_sync(FULL, bmax, kWarp - 1);
      if (!(bm >= sc.strip_floor) || !(bm < sc.strip_ceil)) {
        // (1024: overflowed to inf or NaN, -1024: underflowed to zero)
        strip_lg = (bm != bm || bm >= T(HUGE_VAL)) ? 1024 : (bm > T(0) ? ilogb(bm) : -1024);
        return false;
      }
      strip_lg = ilogb(bm);
      const int ks = sc.target_log2 - strip_lg;
      const int k1 = ks / 2;
      const T f1 = pow2T(k1, T(0)), f2 = pow2T(ks - k1, T(0));
      for (int p = lane; p < S - 1; p += kWarp) {
        T2 v = dst[p];
        v.x = (v.x * f1) * f2;
        v.y = (v.y * f1) * f2;
        dst[p] = v;
      }
      __syncwarp();
      E += ks;
    }
    return true;
  };

  if constexpr (drift) {
    // rescue entries carry one haplotype
    bool ok = K == 1;
    if (nstrips == 1) {
      // a read of one strip: the primary tier (row 0 at 2^120) spilled it because
      // its final sum fell below 2^-80, so it decays by more than 200 bits.  Each
      // lane boosts its own read rows.  The first run spreads 232 bits (32 above
      // that bound) evenly over the read; a run is kept when every lane's
      // bottom-row maximum and the final sum lie in 2^-60 .. 2^60.  Otherwise
      // each lane takes the decay it measured (its boost plus its input's
      // exponent minus its bottom's), so the next run holds every lane near 2^0
      // wherever the read's errors sit.  The first lane whose bottom under- or
      // overflowed moves by the bound that shows (149 bits: a nonzero float would
      // have been seen), and the lanes below it take the mean rate of the lanes
      // above.
      const int used = (n + R - 1) / R;  // lanes holding read rows
      const int lrows = lane < used ? min(R, n - lane * R) : 0;
      const int B0 = min(16 * n, 232);
      lane_boost = true;
      kl_lane = lane < used ? (lane * R + lrows) * B0 / n - (lane * R) * B0 / n : 0;
      for (int attempt = 0; ok; ++attempt) {
        run_strip(std::true_type{}, std::true_type{}, 0, 0);
        const double z = __shfl_sync(FULL, zkeep, kWarp - 1);
        const T lm = lmax_keep;
        const int lgl = lane >= used ? 0 : (lm != lm || lm >= T(HUGE_VAL)) ? 1024 : (lm > T(0) ? ilogb(lm) : -1024);
        const bool in_window = lgl >= -60 && lgl < 60;
        if (__all_sync(FULL, in_window) && z >= (double)sc.final_floor && z < (double)sc.strip_ceil) break;
        if (attempt + 1 == kDriftTries) { ok = false; break; }
        int in = __shfl_up_sync(FULL, lgl, 1);
        if (lane == 0) in = 0;  // row 0 (c = 1)
        const bool measured = lgl > -1024 && lgl < 1024;
        const unsigned bad = __ballot_sync(FULL, lane < used && !measured);
        const int first_bad = bad ? __ffs(bad) - 1 : kWarp;
        const bool valid = lane < used && lane < first_bad;
        const int d = valid ? kl_lane + in - lgl : 0;
        int sum_d = d, sum_r = valid ? lrows : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
          sum_d += __shfl_xor_sync(FULL, sum_d, o);
          sum_r += __shfl_xor_sync(FULL, sum_r, o);
        }
        int k = kl_lane;
        if (valid) {
          k = d;
        } else if (lane < used) {
          if (sum_r > 0) k = (int)((long long)sum_d * lrows / sum_r);
          if (lane == first_bad) k = lgl == -1024 ? max(k, kl_lane + in + 149) : min(k, kl_lane + in - 128);
        }
        kl_lane = max(-24 * lrows, min(24 * lrows, k));
      }
      if (ok) {
        E = kl_lane;
#pragma unroll
        for (int o = 16; o; o >>= 1) E += __shfl_xor_sync(FULL, E, o);
      }
    } else if constexpr (R == kMaxR || R == 4 || R == 2 || R == 1) {
      int Bs = SR;  // first guess: one bit per row (the spilled reads lost more than 160 per strip)
      for (int strip = 0; ok && strip < nstrips; ++strip) {
        const int ns = min(SR, n - strip * SR);
        for (int attempt = 0;; ++attempt) {
          bool good;
          if (strip == 0) {
            good = run_strip(std::true_type{}, std::false_type{}, strip, Bs);
          } else if (strip < nstrips - 1) {
            good = run_strip(std::false_type{}, std::false_type{}, strip, Bs);
          } else {
            run_strip(std::false_type{}, std::true_type{}, strip, Bs);
            const double z = __shfl_sync(FULL, zkeep, kWarp - 1);
            good = z >= (double)sc.final_floor && z < (double)sc.strip_ceil;
            strip_lg = (z != z || z >= HUGE_VAL) ? 1024 : (z > 0.0 ? ilogb(z) : -1024);
          }
          // bottom exponent above the target: the boosts were too strong
          const int excess = strip_lg - sc.target_log2;
          if (good) {
            E += Bs;
            if (strip + 1 < nstrips) {
              // the next strip takes this one's rate plus what it left over
              const int ns1 = min(SR, n - (strip + 1) * SR);
              Bs = max(0, min(16 * ns1, (Bs - excess) * ns1 / ns));
            }
            break;
          }
          if (attempt + 1 == kDriftTries) {
            ok = false;
            break;
          }
          const int step = (strip_lg == 1024) ? -ns / 2 : (strip_lg == -1024) ? ns / 2 : -excess;
          Bs = max(0, min(16 * ns, Bs + (step != 0 ? step : (excess > 0 ? -1 : 1))));
        }
      }
    } else {
      ok = false;  // no strip-mined variant at this R: the pair goes on to FP64
    }
    if (ok && lane == kWarp - 1) {
      const int64_t h = hap_index(0);
      const int m = (int)(bv.hap_off[h + 1] - bv.hap_off[h]);
      bv.out[out_index(0)] = log(zkeep) - (sc.ln_c + log((double)(m + 1))) + lnN - (double)E * kLn2;
    }
    fail = !ok;
  } else if (nstrips == 1) {
    run_strip(std::true_type{}, std::true_type{}, 0, 0);
  } else if constexpr (R == kMaxR || R == 4 || R == 2 || R == 1) {
    bool ok = run_strip(std::true_type{}, std::false_type{}, 0, 0);
    for (int strip = 1; ok && strip < nstrips - 1; ++strip) ok = run_strip(std::false_type{}, std::false_type{}, strip, 0);
    if (ok) ok = run_strip(std::false_type{}, std::true_type{}, nstrips - 1, 0);
    fail = !ok;
  } else {
    fail = true;  // not reached: reads longer than one strip run with R = 8, 4 or 2 (1 in the robust tier)
  }

  if (fail) {
    // a strip underflowed: every pair of this item goes to the next tier
    if (lane == 0) {
      for (int k = 0; k < K; ++k) {
        const int64_t h = hap_index(k);
        const int64_t o = out_index(k);
        if (qv.spill != nullptr) {
          bv.out[o] = __longlong_as_double(0x7ff8000000000000LL);
          spill_pair<T>(qv, w.read, h, o);
        } else {
          bv.out[o] = -HUGE_VAL;
        }
      }
    }
  }
  __syncwarp();
}

// ---- two reads per warp (FP32, semiglobal, one strip) -------------------------
// Two reads of one region with the same rows per lane advance together through
// the region's haplotype stream.  Their rows are packed as float2, so every FMA
// serves both reads (fma.rn.f32x2): per two cells 2 compares, 2 predicated
// multiplies and 4 packed FMAs instead of 12 scalar instructions, and the
// haplotype base load, the ramp and the per-step bookkeeping are shared.
//
// Per row the lane keeps W = x*om + mu of the column it finished -- the
// deletion state om of the NEXT column, computed as soon as mu is known --
// and s; mu itself is not kept.  The next column reads om from W, so the
// arithmetic (and every bit of the result) is that of column(): the same FMA
// on the same operands, one column earlier, and a row holds 2 state words
// instead of 3.
template <int R>
struct PairRows {
  uint32_t ra[R], rb[R];       // read bases of the two reads
  float2 miss[R], K[R], X[R];  // per-row factors (x: first read, y: second)
  float2 W[R], s[R];           // om of the next column, and s, of the column finished last
};

template <int R>
__device__ __forceinline__ void column2(PairRows<R>& w, uint32_t hb, float2 s_top, float2 u_top, float2 k2,
                                        float2 x, float2& u_bot) {
  float2 s_above = s_top;
  float2 nu = u_top;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    float2 mu_new = s_above;
    mul_if_ne(mu_new.x, w.ra[r], hb, w.miss[r].x);
    mul_if_ne(mu_new.y, w.rb[r], hb, w.miss[r].y);
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

__device__ __forceinline__ float2 shfl_up2(float2 v) {
  return make_float2(__shfl_up_sync(0xffffffffu, v.x, 1), __shfl_up_sync(0xffffffffu, v.y, 1));
}

// What a lane needs when it starts haplotype k of a two-read item, written
// once per haplotype by the whole warp into a per-warp ring of kMetaRing
// entries, so the lane that starts it (one lane per step of the ramp) reads
// shared memory instead of a chain of dependent global loads.  A lane starts
// haplotype k at most 31 steps after the warp wrote its entry and lane 31
// finalises it at most 31 steps after that, while the entry is overwritten
// only kMetaRing haplotypes (at least kMetaRing steps) later.
struct HapMeta {
  int64_t ho;     // offset of its bases
  double lnC0;    // ln c + ln(m + 1): the row-0 constant and the free-start count
  int32_t h;      // chunk-local haplotype
  int32_t m;      // length
  int32_t q;      // shared prefix column (-1: none)
  int32_t qn;     // shared prefix column of the next haplotype of the item
  int64_t col;    // output column (added to out_begin / out2_begin)
};
constexpr int kMetaRing = 64;

template <int R>
__device__ __noinline__ void process_pair(const BatchView bv, const QueueView qv, const ItemRef it,
                                          const Tables<float>* __restrict__ tb, const Scalars<float> sc,
                                          const int lane, float4* __restrict__ sv, HapMeta* __restrict__ ring) {
  constexpr unsigned FULL = 0xffffffffu;
  constexpr double kLn2 = 0.6931471805599453094;
  const WorkItem& w = it.w;
  const int64_t offA = bv.read_off[w.read], offB = bv.read_off[w.read2];
  const int nA = (int)(bv.read_off[w.read + 1] - offA);
  const int nB = (int)(bv.read_off[w.read2 + 1] - offB);
  const uint8_t* __restrict__ bA = bv.read_bases + offA;
  const uint8_t* __restrict__ qA = bv.read_quals + offA;
  const uint8_t* __restrict__ bB = bv.read_bases + offB;
  const uint8_t* __restrict__ qB = bv.read_quals + offB;
  const int K = w.nhap;

  double lnA = 0.0, lnB = 0.0;
  for (int i = lane; i < nA; i += kWarp) lnA += tb->lnN[qA[i]];
  for (int i = lane; i < nB; i += kWarp) lnB += tb->lnN[qB[i]];
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    lnA += __shfl_xor_sync(FULL, lnA, o);
    lnB += __shfl_xor_sync(FULL, lnB, o);
  }
  const float AA = tb->A[qA[nA - 1]], AB = tb->A[qB[nB - 1]];
  const float2 k2 = make_float2(sc.k2, sc.k2), x = make_float2(sc.x, sc.x);
  const float2 c2 = make_float2(sc.c, sc.c);
  const bool lane0 = lane == 0;

  // rows as process_item lays out a semiglobal read: the last row's X is
  // alpha*f_n and padding rows pass u down the column
  PairRows<R> rw;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane * R + r;
    if (i < nA) {
      const unsigned q = qA[i];
      rw.ra[r] = bA[i];
      rw.miss[r].x = tb->miss[q];
      rw.K[r].x = tb->K[q];
      rw.X[r].x = (i == nA - 1) ? AA : tb->X[q];
    } else {
      rw.ra[r] = kNeverBase;
      rw.miss[r].x = 0.f;
      rw.K[r].x = 0.f;
      rw.X[r].x = 1.f;
    }
    if (i < nB) {
      const unsigned q = qB[i];
      rw.rb[r] = bB[i];
      rw.miss[r].y = tb->miss[q];
      rw.K[r].y = tb->K[q];
      rw.X[r].y = (i == nB - 1) ? AB : tb->X[q];
    } else {
      rw.rb[r] = kNeverBase;
      rw.miss[r].y = 0.f;
      rw.K[r].y = 0.f;
      rw.X[r].y = 1.f;
    }
    rw.W[r] = make_float2(0.f, 0.f);
    rw.s[r] = make_float2(0.f, 0.f);
  }

  // Shared haplotype prefixes: the item visits its region's haplotypes in
  // lexicographic order (hap_order); when hap_share = Q >= 0 at position k,
  // the haplotype there agrees with the one at k-1 on its first Q bases, so
  // DP columns 0..Q are the same for both.  The lanes lay their state down in
  // shared memory (sv) when they finish column Q at k-1 and start k at column
  // Q+1 from it, so the stream carries only columns Q+1..m.  Lane 31 also
  // carries its row sum across.  The row sums are flushed from FP32 into FP64
  // after every column 8r+7 of lane 31 (by column, not by step), so a shared
  // and an unshared pass give the same bits.
  auto share_of = [&](int k) -> int {
    return (k > 0 && k < K && bv.hap_share != nullptr) ? (int)bv.hap_share[w.hap_begin + k] : -1;
  };
  // haplotype k of the item and its output column: through hap_order when the
  // region's haplotypes are visited in lexicographic order
  auto col_of = [&](int k) -> int64_t {
    return bv.hap_order != nullptr ? (int64_t)bv.hap_order[w.hap_begin + k] : (int64_t)k;
  };
  auto hap_of = [&](int k) -> int64_t {
    return bv.hap_order != nullptr ? (int64_t)bv.hap_order[w.hap_begin + k] : w.hap_begin + k;
  };
  constexpr int kNoSave = INT_MIN;  // no snapshot pending (no stream position, >= -31, matches)
  int kL = -1, next_reset = 0, S_cur = -1, c0 = 0, save_at = kNoSave;
  const uint8_t* hp = bv.hap_bases;
  float2 s_top = make_float2(0.f, 0.f), u_bot = make_float2(0.f, 0.f), acc32 = make_float2(0.f, 0.f);
  double accA = 0.0, accB = 0.0;
  // snapshot layout, 16-byte entries slot-major with one entry per lane (the
  // lane that saves or restores is alone in its branch, so its instruction
  // count is what costs): (W, s) of each row, (s_top, FP32 row sums), the two
  // FP64 row sums
  double2* const svd = reinterpret_cast<double2*>(sv + (R + 1) * kWarp);

  // the warp writes haplotype k's ring entry (every lane computes it, lane 0
  // stores it)
  auto publish = [&](int k) -> HapMeta {
    HapMeta e;
    e.h = (int32_t)hap_of(k);
    e.ho = bv.hap_off[e.h];
    e.m = (int32_t)(bv.hap_off[e.h + 1] - e.ho);
    e.q = share_of(k);
    e.qn = share_of(k + 1);
    e.col = col_of(k);
    e.lnC0 = sc.ln_c + log((double)(e.m + 1));
    if (lane == 0) ring[k & (kMetaRing - 1)] = e;
    __syncwarp();
    return e;
  };

  auto finalize = [&](int k) {
    const HapMeta& e = ring[k & (kMetaRing - 1)];
    const int64_t h = e.h;
    const double lnC0 = e.lnC0;
    const double za = accA + (double)acc32.x, zb = accB + (double)acc32.y;
    const int64_t oa = w.out_begin + e.col, ob = w.out2_begin + e.col;
    if (za >= (double)sc.final_floor && za < HUGE_VAL) {
      bv.out[oa] = log(za) - lnC0 + lnA;
    } else {
      bv.out[oa] = __longlong_as_double(0x7ff8000000000000LL);
      spill_pair<float>(qv, w.read, h, oa);
    }
    if (zb >= (double)sc.final_floor && zb < HUGE_VAL) {
      bv.out[ob] = log(zb) - lnC0 + lnB;
    } else {
      bv.out[ob] = __longlong_as_double(0x7ff8000000000000LL);
      spill_pair<float>(qv, w.read2, h, ob);
    }
  };

  auto flush = [&]() {
    accA += (double)acc32.x;
    accB += (double)acc32.y;
    acc32 = make_float2(0.f, 0.f);
  };
  auto save = [&]() {
#pragma unroll
    for (int r = 0; r < R; ++r) sv[r * kWarp + lane] = make_float4(rw.W[r].x, rw.W[r].y, rw.s[r].x, rw.s[r].y);
    sv[R * kWarp + lane] = make_float4(s_top.x, s_top.y, acc32.x, acc32.y);
    svd[lane] = make_double2(accA, accB);
  };
  auto restore = [&]() {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const float4 v = sv[r * kWarp + lane];
      rw.W[r] = make_float2(v.x, v.y);
      rw.s[r] = make_float2(v.z, v.w);
    }
    const float4 v = sv[R * kWarp + lane];
    s_top = make_float2(v.x, v.y);
    acc32 = make_float2(v.z, v.w);
    const double2 a = svd[lane];
    accA = a.x;
    accB = a.y;
  };

  // step with per-lane haplotype bookkeeping (ramps, snapshots, short haplotypes)
  auto gstep = [&](int t) {
    const int p = t - lane;
    float2 u_in = shfl_up2(u_bot);
    float2 s_in = shfl_up2(rw.s[R - 1]);
    if (p == next_reset) {
      if (kL >= 0 && lane == kWarp - 1) finalize(kL);
      ++kL;
      S_cur = p;
      save_at = kNoSave;
      if (kL < K) {
        const HapMeta& e = ring[kL & (kMetaRing - 1)];
        const int q = e.q;
        c0 = q + 1;
        if (q >= 0) {
          restore();
        } else {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            rw.W[r] = make_float2(0.f, 0.f);
            rw.s[r] = make_float2(0.f, 0.f);
          }
          s_top = make_float2(0.f, 0.f);
          acc32 = make_float2(0.f, 0.f);
          accA = accB = 0.0;
        }
        hp = bv.hap_bases + e.ho + c0 - 1 - p;
        next_reset = p + e.m + 1 - c0;
        // the next haplotype starts from column qn: a snapshot of it is taken
        // here, or (qn == c0 - 1) the one this haplotype started from stays
        const int qn = e.qn;
        if (qn >= c0) save_at = p + (qn - c0);
      } else {
        next_reset = INT_MAX;
      }
    }
    const bool active = kL >= 0 && kL < K;
    const uint32_t hb = (active && !(p == S_cur && c0 == 0)) ? (uint32_t)hp[p] : 0u;
    u_in = lane0 ? c2 : u_in;
    s_in = lane0 ? c2 : s_in;
    column2<R>(rw, hb, s_top, u_in, k2, x, u_bot);
    s_top = s_in;
    acc32 = __fadd2_rn(acc32, u_bot);
    // lane 31 alone flushes, after its columns 8r+7
    if (lane == kWarp - 1 && ((c0 + p - S_cur) & 7) == 7) flush();
    if (p == save_at) save();
  };

  // step with every lane inside the same haplotype past its start column
  auto sstep = [&](uint32_t hb) {
    float2 u_in = shfl_up2(u_bot);
    float2 s_in = shfl_up2(rw.s[R - 1]);
    u_in = lane0 ? c2 : u_in;
    s_in = lane0 ? c2 : s_in;
    column2<R>(rw, hb, s_top, u_in, k2, x, u_bot);
    s_top = s_in;
    acc32 = __fadd2_rn(acc32, u_bot);
  };

  int t = 0, S = 0;
  for (int k = 0; k <= K; ++k) {
    int seg = 0, ck = 0, w0 = -1;
    if (k < K) {
      const HapMeta e = publish(k);
      ck = e.q + 1;
      seg = e.m + 1 - ck;
      if (e.qn >= ck) w0 = S + (e.qn - ck);  // lanes take the snapshot at steps w0 .. w0 + 31
    }
    const int Snext = S + seg;
    const int gen_end = (k < K) ? min(S + kWarp, Snext) : S + kWarp;
    for (; t < gen_end; ++t) gstep(t);
    if (k < K) {
      // all lanes are inside haplotype k for t in [S + 32, Snext); the
      // snapshot window of the next haplotype runs through gstep
      while (t < Snext) {
        if (w0 >= 0 && t >= w0 && t < w0 + kWarp) {
          // no lane starts a haplotype here: a column step, lane 31's flush
          // by column and the snapshot of the lane whose turn it is
          sstep((uint32_t)hp[t - lane]);
          if (((ck - (kWarp - 1) - S + t) & 7) == 7) flush();
          if (t - lane == save_at) save();
          ++t;
          continue;
        }
        const int stop = (w0 >= 0 && t < w0) ? min(w0, Snext) : Snext;
        // lane 31's column at step t is ck + (t - 31 - S); single steps bring
        // it to a multiple of 8, so every block of 8 ends on a column 8r+7
        const int lead = ck - (kWarp - 1) - S;
        for (; t < stop && ((lead + t) & 7) != 0; ++t) {
          sstep((uint32_t)hp[t - lane]);
          if (((lead + t) & 7) == 7) flush();
        }
        static_assert(kUnroll == 8, "blocks of 8 steps flush once, at their last column");
        for (; t + kUnroll <= stop; t += kUnroll) {
          const uint8_t* q = hp + (t - lane);
#pragma unroll
          for (int u = 0; u < kUnroll; ++u) sstep((uint32_t)q[u]);
          flush();
        }
        for (; t < stop; ++t) sstep((uint32_t)hp[t - lane]);  // columns 8r..8r+6: no flush
      }
    }
    S = Snext;
  }
  __syncwarp();
}

template <typename T, bool ANCH>
__device__ __forceinline__ void dispatch(int code, const BatchView& bv, const QueueView& qv,
                                         const ItemRef& it, const Tables<T>* tb, const Scalars<T>& sc,
                                         int lane, typename Vec2<T>::type* scratch) {
  const bool gen = code_general(code);
#define VD_CASE(r)                                                                   \
  case r:                                                                            \
    if (gen) process_item<T, r, true, ANCH>(bv, qv, it, tb, sc, lane, scratch);      \
    else process_item<T, r, false, ANCH>(bv, qv, it, tb, sc, lane, scratch);         \
    break;
  switch (code_R(code)) {
    VD_CASE(1) VD_CASE(2) VD_CASE(3) VD_CASE(4) VD_CASE(5) VD_CASE(6) VD_CASE(7) VD_CASE(8)
    default: break;
  }
#undef VD_CASE
}

// Persistent kernel: every warp pulls work from qv.head until the list is
// exhausted.  tier 0 reads WorkItems; tiers 1 and 2 read the rescue list the
// previous tier spilled (one haplotype per entry).  Tier 2 runs R = 1 (strips
// of 32 rows, renormalised between strips), which no input can underflow.
// Resident blocks per SM the compiler must fit: the FP32 kernel is issue
// bound and gains from 20 warps per SM (96 registers); the FP64 tiers run
// 12 warps per SM (168 registers), 4% faster on error-rich 1-10 kb reads
// than 8 warps with no spills.
template <typename T> struct MinBlocks { static constexpr int value = 1; };
template <> struct MinBlocks<float> { static constexpr int value = 5; };
template <> struct MinBlocks<double> { static constexpr int value = 3; };

template <typename T, bool ANCH>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp, MinBlocks<T>::value)
pairhmm_kernel(const BatchView bv, const QueueView qv, const Tables<T>* __restrict__ gtab,
               const Scalars<T> sc, const int tier) {
  __shared__ Tables<T> tab;
  {
    const int words = (int)(sizeof(Tables<T>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(gtab);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  using T2 = typename Vec2<T>::type;
  const int lane = threadIdx.x & (kWarp - 1);
  const long long gw = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  T2* scratch = reinterpret_cast<T2*>(qv.scratch) + gw * qv.scratch_stride;
  // primary tier: n_items work items; rescue tiers: the count the previous
  // tier spilled, bounded by the capacity of its list (n_items)
  long long total = qv.n_items;
  if (qv.items == nullptr) {
    const long long c = (long long)*qv.count;
    total = c < total ? c : total;
  }
  // the plain schedule walks the list in a fixed round-robin order; the
  // batched one pulls items from the shared counter
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
    if ((long long)i >= total) break;
    ItemRef it;
    it.tier = tier;
    int code;
    if (qv.items != nullptr) {
      it.w = qv.items[i];
      it.use_sel = bv.hap_sel != nullptr;
      code = it.w.code;
    } else {
      const RescueEntry e = qv.entries[i];
      it.w.read = e.read;
      it.w.nhap = 1;
      it.w.hap_begin = e.hap;
      it.w.out_begin = e.out;
      it.w.read2 = -1;
      it.w.out2_begin = 0;
      it.use_sel = false;
      const int rc = bv.read_code[e.read];
      code = (tier >= 2) ? make_code(1, code_general(rc), true) : rc;
      it.w.code = code;
    }
    dispatch<T, ANCH>(code, bv, qv, it, &tab, sc, lane, scratch);
  }
}

// Persistent kernels of the two-read items (FP32, semiglobal), on their own
// work list ahead of the single-read items of the same tier.  Packed rows
// need about 12 registers each: items with 6-8 rows per lane run 3 blocks per
// SM (168 registers), items with up to 5 rows 4 blocks (128 registers), each
// kernel instantiating only its own row counts.  (Resident warps come in
// steps of 4 per SM whatever the block size: each of the 4 schedulers holds
// a quarter of the register file, so 13-15 warps need no more than 128
// registers either.)
template <int kLoR, int kHiR, int kBlocks, int kWarps = kWarpsPerBlock>
__global__ void __launch_bounds__(kWarps * kWarp, kBlocks)
pairhmm_pair_kernel(const BatchView bv, const QueueView qv, const Tables<float>* __restrict__ gtab,
                    const Scalars<float> sc) {
  __shared__ Tables<float> tab;
  // per warp: the lane states laid down at a shared haplotype prefix
  __shared__ float4 saves[kWarps][(kHiR + 2) * kWarp];
  __shared__ HapMeta meta[kWarps][kMetaRing];
  {
    const int words = (int)(sizeof(Tables<float>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(gtab);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1);
  float4* sv = saves[threadIdx.x >> 5];
  for (;;) {
    unsigned long long i = 0;
    if (lane == 0) i = atomicAdd(qv.head, 1ull);
    i = __shfl_sync(0xffffffffu, i, 0);
    if ((long long)i >= qv.n_items) break;
    ItemRef it;
    it.w = qv.items[i];
    it.use_sel = false;
    it.tier = 0;
    switch (code_R(it.w.code)) {
#define VD_PCASE(r) \
      case r: if constexpr (r >= kLoR && r <= kHiR) process_pair<r>(bv, qv, it, &tab, sc, lane, sv, meta[threadIdx.x >> 5]); break;
      VD_PCASE(1) VD_PCASE(2) VD_PCASE(3) VD_PCASE(4) VD_PCASE(5) VD_PCASE(6) VD_PCASE(7) VD_PCASE(8)
#undef VD_PCASE
      default: break;
    }
  }
}

// The drift tier (FP32, semiglobal): the rescue list of the primary tier,
// each entry in the two-sided emission form its boosted match factors need,
// on its own kernel so the strip driver's state does not crowd the primary
// kernel's registers (launched with 4 blocks per SM, 128 registers: 7% faster
// on the mixed-length workload's long reads than 3 blocks at 162 registers without spills).
// Reads of one strip run at their own rows per lane; longer reads whose rows
// per lane have no strip-mined variant go on to FP64 unchanged.
template <int kBlocks>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp, kBlocks)
pairhmm_drift_kernel(const BatchView bv, const QueueView qv, const Tables<float>* __restrict__ gtab,
                     const Scalars<float> sc) {
  __shared__ Tables<float> tab;
  {
    const int words = (int)(sizeof(Tables<float>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(gtab);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & (kWarp - 1);
  const long long gw = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  float2* scratch = reinterpret_cast<float2*>(qv.scratch) + gw * qv.scratch_stride;
  long long total = qv.n_items;
  const long long c = (long long)*qv.count;
  total = c < total ? c : total;
  for (;;) {
    unsigned long long i = 0;
    if (lane == 0) i = atomicAdd(qv.head, 1ull);
    i = __shfl_sync(0xffffffffu, i, 0);
    if ((long long)i >= total) break;
    const RescueEntry e = qv.entries[i];
    ItemRef it;
    it.tier = kDriftTier;
    it.use_sel = false;
    it.w.read = e.read;
    it.w.nhap = 1;
    it.w.hap_begin = e.hap;
    it.w.out_begin = e.out;
    it.w.read2 = -1;
    it.w.out2_begin = 0;
    it.w.code = bv.read_code[e.read];
    switch (code_R(it.w.code)) {
#define VD_DCASE(r) \
      case r: process_item<float, r, true, false, true>(bv, qv, it, &tab, sc, lane, scratch); break;
      VD_DCASE(1) VD_DCASE(2) VD_DCASE(3) VD_DCASE(4) VD_DCASE(5) VD_DCASE(6) VD_DCASE(7) VD_DCASE(8)
#undef VD_DCASE
      default:
        if (lane == 0) spill_pair<float>(qv, e.read, e.hap, e.out);
        __syncwarp();
        break;
    }
  }
}

}  // namespace vd
