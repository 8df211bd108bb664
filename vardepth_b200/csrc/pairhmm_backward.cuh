// Reverse-wavefront gradient of the PairHMM log-likelihood on sm_100a.
//
// For every read x haplotype pair the kernel returns ln L and the six partial
// derivatives d ln L / d theta, theta = (gap-open Phred Qg, gap-continuation
// Phred Qx, Phred offsets o0..o3 of the four quality bins), g = 10^(-Qg/10),
// x = 10^(-Qx/10), e = 10^(-max(0, min(q,60) + o_bin(q))/10).  The reference
// has no differentiable PairHMM: this is reverse-mode differentiation of the
// scaled forward recurrence of pairhmm_core.cuh, i.e. (semiglobal mode) of
//   mu_i(j) = s_{i-1}(j-1) h_ij                 h = hit or miss of row i
//   om_i(j) = mu_i(j-1) + x om_i(j-1)
//   u_i(j)  = mu_i(j) + X_i u_{i-1}(j)          (X_n = A_n on the last row)
//   s_i(j)  = mu_i(j) + K_i u_{i-1}(j) + k2 om_i(j)
//   Zs = sum_j u_n(j),  ln L = ln Zs - ln c - ln(m+1) + sum_i ln N_i.
// Its adjoint (~ marks dZs/d(variable), scaled by a power of two rho):
//   s~_i(j)  = h_{i+1,j+1} mu~_{i+1}(j+1)
//   u~_i(j)  = X_{i+1} u~_{i+1}(j) + K_{i+1} s~_{i+1}(j)      (u~_n = rho)
//   om~_i(j) = k2 s~_i(j) + x om~_i(j+1)
//   mu~_i(j) = u~_i(j) + s~_i(j) + om~_i(j+1)
// and every folded constant collects (adjoint of its product) x (its operand):
//   per row  pu = sum_j u~ nu,  ps = sum_j s~ nu,  bM = sum_{mismatch} mu~ mu,
//            bH = sum_{match} mu~ mu (two-sided rows only)
//   global   Bk2 = sum s~ om,  Ax = sum om~_i(j+1) om_i(j)
// so that with the log-derivative tables of the constants (GradTables)
//   d ln L = [sum_rows (X pu dlnX + K ps dlnK + bM dlnmiss + bH dlnhit)
//             + k2 Bk2 dlnk2 + Ax dx] / (rho Zs) + sum_rows dlnN.
// Anchored mode differentiates Zs = (mu + A nu + g om)_n(m), the end cell, with
// the virtual row-0 emulator of the forward kernel; the end cell seeds the
// adjoint (mu~ = rho, om~ = rho g, and rho A into u~ of the row above) and A
// and g collect rho A nu and rho g om there.
//
// Layout: one warp per pair, lane L owns R consecutive rows (reads of at
// most 256 bases, one strip), the anti-diagonal sweep of the forward kernel.
// The reverse sweep runs the steps backwards: lane L takes the adjoint of the
// row below from lane L+1 by __shfl_down_sync (u~ at the same column, s~ one
// column to the right, held for a step), the mirror image of the forward.
//
// Memory: the forward values a backward step needs (mu and omega of the
// lane's rows and the u handed in from the row above: 2R+1 values per lane
// and step) are produced by recomputation.  A first forward pass stores the
// warp state every C steps (C = ceil(sqrt(T)) for T = m + 33 steps, "sqrt-L
// anti-diagonal checkpointing"); the reverse sweep replays each segment of C
// steps from its checkpoint once to lay down a state every kSub = 6 steps,
// then replays each 6-step sub-segment into a shared-memory buffer and walks
// it back from there, so the per-step values never leave the SM.  With
// store_all the first pass keeps every step in global memory (one segment of
// T steps).  Both give bit-identical results.
#pragma once
#include "pairhmm_kernel.cuh"

namespace vd {

// Derivatives of the per-quality constants with respect to the offset of the
// quality's bin, in Phred units (0 where the Phred floor at 0 binds).
struct GradTables {
  double dlnN[256];     // d ln N_q / d o
  double dlnmiss[256];  // d ln miss_q / d o
  double dlnhit[256];   // d ln hit_q / d o (two-sided rows)
  int bin[256];         // quality bin of the Phred byte
};

// Derivatives with respect to Qg and Qx, identical for every row.
struct GradScalars {
  double dlnN_g, dlnK_g, dlnX_g, dlnA_g, dlnk2_g, dlng_g;
  double dlnK_x, dlnX_x, dlnk2_x, dx_x;
};

struct GradView {
  const RescueEntry* items;          // (read, hap, out) per pair
  const unsigned long long* count;   // nullable: items to take from a device counter
  long long n_items;
  unsigned long long* head;
  double* out_ln;                    // per output slot
  double* out_jac;                   // per output slot, 6 doubles
  char* scratch;                     // per warp slot: checkpoints and the segment buffer
  long long slot_bytes;
  int store_all;
  int anchored;                      // 0: semiglobal, 1: anchored (global) model
  RescueEntry* spill;                // FP32 pass: pairs left to the FP64 pass
  unsigned long long* spill_count;
  long long spill_cap;
  int* error_flag;                   // bit 0: spill overflow, bit 1: an FP64 pair underflowed
};

// Steps of one pair's wavefront and its checkpoint interval; shared with the
// host, which sizes the scratch from it.
__host__ __device__ inline int grad_steps(int m) { return m + kWarp + 1; }
__host__ __device__ inline int grad_interval(int steps, bool store_all) {
  if (store_all) return steps;
  int c = (int)ceil(sqrt((double)steps));
  return c < 4 ? 4 : c;
}
// Steps of the shared-memory sub-segment buffer (sqrt-L mode): each sqrt(T)
// segment is replayed once to lay down a warp state every kSub steps, then
// sub-segment by sub-segment into shared memory and walked back from there.
constexpr int kSub = 6;
// Shared memory of one warp's sub-segment buffer, sized for R = 8.
template <typename T>
__host__ __device__ constexpr int grad_smem_per_warp() { return kSub * (2 * kMaxR + 1) * kWarp * (int)sizeof(T); }
// Elements of type T one warp slot needs in global memory for a pair with R
// rows per lane: the sqrt(T) checkpoints and the sub-segment states, or every
// step's buffer row when store_all.
__host__ __device__ inline long long grad_slot_elems(int R, int m, bool store_all) {
  const int steps = grad_steps(m);
  const int C = grad_interval(steps, store_all);
  const int nseg = (steps + C - 1) / C;
  if (store_all) return (long long)C * (2 * R + 1) * kWarp;
  return ((long long)nseg + (C + kSub - 1) / kSub) * (3 * R + 2) * kWarp;
}

// The adjoint starts at rho = 2^k on the last row, with rho Zs near 2^kTarget
// (k at most kMax): on the most likely path the forward values fall from c at
// the top row towards Zs and the adjoint falls from rho at the bottom towards
// rho Zs / c, so the products stay near rho Zs and the adjoint keeps the
// exponent range below it for paths away from the most likely one.
template <typename T> struct GradConsts { static constexpr int kTarget = 100, kMax = 120; };
template <> struct GradConsts<double> { static constexpr int kTarget = 600, kMax = 900; };

template <typename T, int R, bool GEN, bool ANCH>
__device__ __noinline__ void grad_pair(const BatchView& bv, const GradView& gv, const RescueEntry item,
                                       const Tables<T>* __restrict__ tb, const Scalars<T>& sc,
                                       const GradTables* __restrict__ gt, const GradScalars& gs, const int lane,
                                       T* __restrict__ slot, T* __restrict__ sbuf) {
  constexpr unsigned FULL = 0xffffffffu;
  const int64_t roff = bv.read_off[item.read];
  const int n = (int)(bv.read_off[item.read + 1] - roff);
  const uint8_t* __restrict__ rbase = bv.read_bases + roff;
  const uint8_t* __restrict__ rqual = bv.read_quals + roff;
  const int64_t hoff = bv.hap_off[item.hap];
  const int m = (int)(bv.hap_off[item.hap + 1] - hoff);
  const uint8_t* __restrict__ hap = bv.hap_bases + hoff;
  const int64_t o = item.out;

  const bool store_all = gv.store_all != 0;
  const int steps = grad_steps(m);
  const int C = grad_interval(steps, store_all);
  const int nseg = (steps + C - 1) / C;
  constexpr int CKW = 3 * R + 2;  // checkpoint words per lane
  constexpr int BFW = 2 * R + 1;  // segment-buffer words per lane and step
  T* __restrict__ ck = slot;                                   // sqrt(T) checkpoints
  T* __restrict__ sub = slot + (long long)nseg * CKW * kWarp;   // states every kSub steps of a segment
  T* __restrict__ buf = slot;                                  // store_all: every step

  const T k2 = sc.k2, x = sc.x, c0 = sc.c, gfin = sc.gfin;
  const T A = tb->A[rqual[n - 1]];

  // rows of this lane: the layout of process_item for one strip.  Semiglobal:
  // row i = 32 lane ... with padding rows below the read passing u down.
  // Anchored: the read is bottom-aligned below v = 32 R - n virtual rows, the
  // lowest of them (i = -1) the emulator of row 0, fed s(-1) = c at column 0.
  const int v = ANCH ? kWarp * R - n : 0;
  int emu = -1;
  LaneRows<T, R, GEN> rw;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane * R + r - v;
    if (i >= 0 && i < n) {
      const unsigned q = rqual[i];
      rw.rb[r] = rbase[i];
      rw.miss[r] = tb->miss[q];
      if (GEN) rw.hit[r] = tb->hit[q];
      rw.K[r] = tb->K[q];
      rw.X[r] = (!ANCH && i == n - 1) ? A : tb->X[q];
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
  T s_top = T(0), u_bot = T(0);
  double acc = 0.0;
  // anchored end cell: (M + I + D)[n][m] = mu + A nu + g om of the last row at
  // column m, the running maximum of that sum over the row (the 1e-300 floor of
  // anchored.cpp:24), and its nu and om (the operands of A and g in it)
  T cap = T(0), rmax = T(0), end_nu = T(0), end_om = T(0);

  // one forward step; with rec the lane's column values go to row t - t0 of
  // dst (the global buffer, or this warp's shared sub-segment buffer)
  auto fstep = [&](const int t, const int t0, const bool rec, T* __restrict__ dst) {
    const int j = t - lane;
    T u_in = __shfl_up_sync(FULL, u_bot, 1);
    T s_in = __shfl_up_sync(FULL, rw.s[R - 1], 1);
    if (lane == 0) { u_in = ANCH ? T(0) : c0; s_in = u_in; }
    if (j == 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) { rw.mu[r] = T(0); rw.om[r] = T(0); rw.s[r] = T(0); }
      s_top = T(0);
      if (ANCH) {
        if (emu == 0) s_top = c0;
#pragma unroll
        for (int r = 1; r < R; ++r)
          if (emu == r) rw.s[r - 1] = c0;
      }
    }
    const bool act = (unsigned)j <= (unsigned)m;
    const uint32_t hb = (act && j > 0) ? (uint32_t)hap[j - 1] : 0u;
    T tmu = T(0), tnu = T(0), tom = T(0);
    column<T, R, GEN, ANCH>(rw, hb, s_top, u_in, k2, x, u_bot, tmu, tnu, tom);
    s_top = s_in;
    if (rec && act) {
      T* e = dst + (long long)(t - t0) * BFW * kWarp + lane;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        e[r * kWarp] = rw.mu[r];
        e[(R + r) * kWarp] = rw.om[r];
      }
      e[2 * R * kWarp] = u_in;
    }
    if (lane == kWarp - 1 && act) {
      if (ANCH) {
        cap = fmaT(gfin, tom, fmaT(A, tnu, tmu));
        rmax = maxT(rmax, cap);
        if (j == m) { end_nu = tnu; end_om = tom; }
      } else {
        acc += (double)u_bot;
      }
    }
  };
  auto save_state = [&](T* __restrict__ area, const int k) {
    T* e = area + (long long)k * CKW * kWarp + lane;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      e[r * kWarp] = rw.mu[r];
      e[(R + r) * kWarp] = rw.om[r];
      e[(2 * R + r) * kWarp] = rw.s[r];
    }
    e[3 * R * kWarp] = s_top;
    e[(3 * R + 1) * kWarp] = u_bot;
  };
  auto load_state = [&](const T* __restrict__ area, const int k) {
    const T* e = area + (long long)k * CKW * kWarp + lane;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rw.mu[r] = e[r * kWarp];
      rw.om[r] = e[(R + r) * kWarp];
      rw.s[r] = e[(2 * R + r) * kWarp];
    }
    s_top = e[3 * R * kWarp];
    u_bot = e[(3 * R + 1) * kWarp];
  };

  // ---- first forward pass: Zs, and the checkpoints (or every step) ----
  for (int t = 0; t < steps; ++t) {
    if (!store_all && t % C == 0) save_state(ck, t / C);
    fstep(t, 0, store_all, buf);
  }
  const double Zs = __shfl_sync(FULL, ANCH ? (double)cap : acc, kWarp - 1);
  const double Zmax = __shfl_sync(FULL, (double)rmax, kWarp - 1);
  double lnN = 0.0;
  for (int i = lane; i < n; i += kWarp) lnN += tb->lnN[rqual[i]];
#pragma unroll
  for (int s = 16; s; s >>= 1) lnN += __shfl_xor_sync(FULL, lnN, s);
  const bool ok = Zs >= (double)sc.final_floor && Zs < HUGE_VAL;
  if (!ok) {
    // the FP32 pass hands the pair to the FP64 pass; an FP64 failure is flagged
    if (lane == 0) {
      const double nan = __longlong_as_double(0x7ff8000000000000LL);
      gv.out_ln[o] = nan;
      for (int k = 0; k < 6; ++k) gv.out_jac[o * 6 + k] = nan;
      if (gv.spill != nullptr) {
        const unsigned long long s = atomicAdd(gv.spill_count, 1ull);
        if ((long long)s < gv.spill_cap) gv.spill[s] = item;
        else atomicOr(gv.error_flag, 1);
      } else {
        atomicOr(gv.error_flag, 2);
      }
    }
    __syncwarp();
    return;
  }

  // ---- reverse sweep ----
  const int rho_log2 = min(GradConsts<T>::kMax, GradConsts<T>::kTarget - ilogb(Zs));
  const T rho = pow2T(rho_log2, T(0));
  T ome[R], ups[R], pu[R], ps[R], bM[R], bH[GEN ? R : 1];
#pragma unroll
  for (int r = 0; r < R; ++r) { ome[r] = T(0); ups[r] = T(0); pu[r] = T(0); ps[r] = T(0); bM[r] = T(0); }
#pragma unroll
  for (int r = 0; r < (GEN ? R : 1); ++r) bH[r] = T(0);
  T Bk2 = T(0), Ax = T(0);
  T top_u = T(0), top_s = T(0), pend_s = T(0);

  auto bstep = [&](const int t, const int t0, const T* __restrict__ src) {
    const int j = t - lane;
    const bool act = (unsigned)j <= (unsigned)m;
    T in_u = __shfl_down_sync(FULL, top_u, 1);
    T in_s_next = __shfl_down_sync(FULL, top_s, 1);
    // semiglobal: every (M + I)[n][j] is summed, so u of the bottom row has
    // adjoint rho; anchored: only the end cell counts (seeded below)
    if (lane == kWarp - 1) { in_u = (act && !ANCH) ? rho : T(0); in_s_next = T(0); }
    // anchored end cell at column m: d/dmu = rho, d/dom = rho g, d/dnu = rho A
    const bool seed = ANCH && lane == kWarp - 1 && j == m;
    const T in_s = pend_s;
    pend_s = in_s_next;
    if (!act) {
      top_u = T(0);
      top_s = T(0);
      return;
    }
    const T* e = src + (long long)(t - t0) * BFW * kWarp + lane;
    T muf[R], omf[R], nu[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      muf[r] = e[r * kWarp];
      omf[r] = e[(R + r) * kWarp];
    }
    nu[0] = e[2 * R * kWarp];
#pragma unroll
    for (int r = 1; r < R; ++r) nu[r] = fmaT(rw.X[r - 1], nu[r - 1], muf[r - 1]);
    const uint32_t hb = j > 0 ? (uint32_t)hap[j - 1] : 0u;
    T cu = in_u, cs = in_s;
#pragma unroll
    for (int r = R - 1; r >= 0; --r) {
      const T sb = cs, ub = cu;
      const bool sd = seed && r == R - 1;
      const T omb = fmaT(x, ome[r], k2 * sb) + (sd ? rho * gfin : T(0));
      const T mub = ub + sb + ome[r] + (sd ? rho : T(0));
      pu[r] = fmaT(ub, nu[r], pu[r]);
      ps[r] = fmaT(sb, nu[r], ps[r]);
      const bool match = rw.rb[r] == hb;
      T up_s;
      if (GEN) {
        if (match) bH[r] = fmaT(mub, muf[r], bH[r]);
        else bM[r] = fmaT(mub, muf[r], bM[r]);
        up_s = mub * (match ? rw.hit[r] : rw.miss[r]);
      } else {
        bM[r] = fmaT(match ? T(0) : mub, muf[r], bM[r]);
        up_s = match ? mub : mub * rw.miss[r];
      }
      Bk2 = fmaT(sb, omf[r], Bk2);
      Ax = fmaT(ome[r], omf[r], Ax);
      ome[r] = omb;
      cu = fmaT(rw.X[r], ub, rw.K[r] * sb) + (sd ? rho * A : T(0));
      cs = ups[r];
      ups[r] = up_s;
    }
    top_u = cu;
    top_s = ups[0];
  };

  if (store_all) {
    __syncwarp();
    for (int t = steps - 1; t >= 0; --t) bstep(t, 0, buf);
    __syncwarp();
  } else {
    for (int k = nseg - 1; k >= 0; --k) {
      const int t0 = k * C;
      const int t1 = min(steps, t0 + C);
      // lay down a state every kSub steps of the segment, then walk the
      // sub-segments back through shared memory
      load_state(ck, k);
      for (int t = t0; t < t1; ++t) {
        if ((t - t0) % kSub == 0) save_state(sub, (t - t0) / kSub);
        fstep(t, t0, false, buf);
      }
      __syncwarp();
      for (int q = (t1 - t0 - 1) / kSub; q >= 0; --q) {
        const int ta = t0 + q * kSub;
        const int tb = min(t1, ta + kSub);
        load_state(sub, q);
        for (int t = ta; t < tb; ++t) fstep(t, ta, true, sbuf);
        __syncwarp();
        for (int t = tb - 1; t >= ta; --t) bstep(t, ta, sbuf);
        __syncwarp();
      }
    }
  }

  // ---- chain rule to theta (FP64) ----
  const double inv = 1.0 / (ldexp(1.0, rho_log2) * Zs);
  double jg = 0.0, jx = 0.0, jo0 = 0.0, jo1 = 0.0, jo2 = 0.0, jo3 = 0.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane * R + r - v;
    if (i >= 0 && i < n) {
      const unsigned q = rqual[i];
      const bool last = !ANCH && i == n - 1;
      const double bX = (double)rw.X[r] * (double)pu[r];
      const double bK = (double)rw.K[r] * (double)ps[r];
      jg += (bX * (last ? gs.dlnA_g : gs.dlnX_g) + bK * gs.dlnK_g) * inv + gs.dlnN_g;
      jx += (bX * (last ? 0.0 : gs.dlnX_x) + bK * gs.dlnK_x) * inv;
      const double bh = GEN ? (double)bH[r] : 0.0;
      const double d = ((double)bM[r] * gt->dlnmiss[q] + bh * gt->dlnhit[q] - (bX + bK) * gt->dlnN[q]) * inv +
                       gt->dlnN[q];
      const int b = gt->bin[q];
      jo0 += b == 0 ? d : 0.0;
      jo1 += b == 1 ? d : 0.0;
      jo2 += b == 2 ? d : 0.0;
      jo3 += b == 3 ? d : 0.0;
    }
  }
  jg += (double)k2 * (double)Bk2 * gs.dlnk2_g * inv;
  jx += ((double)k2 * (double)Bk2 * gs.dlnk2_x + (double)Ax * gs.dx_x) * inv;
  if (ANCH && lane == kWarp - 1) {
    // the end cell's own constants: A = (g/4) f_n and g (d ln g / dQg = -ln(10)/10)
    const double rho_d = ldexp(1.0, rho_log2);
    const double bA = rho_d * (double)A * (double)end_nu, bg = rho_d * (double)gfin * (double)end_om;
    const unsigned q = rqual[n - 1];
    jg += (bA * gs.dlnA_g + bg * gs.dlng_g) * inv;
    const double d = -bA * gt->dlnN[q] * inv;
    const int b = gt->bin[q];
    jo0 += b == 0 ? d : 0.0;
    jo1 += b == 1 ? d : 0.0;
    jo2 += b == 2 ? d : 0.0;
    jo3 += b == 3 ? d : 0.0;
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    jg += __shfl_xor_sync(FULL, jg, s);
    jx += __shfl_xor_sync(FULL, jx, s);
    jo0 += __shfl_xor_sync(FULL, jo0, s);
    jo1 += __shfl_xor_sync(FULL, jo1, s);
    jo2 += __shfl_xor_sync(FULL, jo2, s);
    jo3 += __shfl_xor_sync(FULL, jo3, s);
  }
  if (lane == 0) {
    const double lnC0 = (double)sc.ln_c + (ANCH ? 0.0 : log((double)(m + 1)));
    // anchored.cpp:24 floors the end cell at 1e-300 of the last row's maximum;
    // the gradient is that of the unfloored value
    const double Zc = ANCH ? fmax(Zs, 1e-300 * Zmax) : Zs;
    gv.out_ln[o] = log(Zc) - lnC0 + lnN;
    double* J = gv.out_jac + o * 6;
    J[0] = jg;
    J[1] = jx;
    J[2] = jo0;
    J[3] = jo1;
    J[4] = jo2;
    J[5] = jo3;
  }
  __syncwarp();
}

// Persistent gradient kernel: warps pull pairs from gv.head.  The FP32 pass
// reads the host-built list; the FP64 pass reads what the FP32 pass spilled.
// Blocks per SM: the FP32 pass fits three (168 registers, 3 x 67 KB of shared
// memory with 6-step buffers), 18% faster than two at 178 registers; the FP64
// pass keeps its registers.
template <typename T> struct GradMinBlocks { static constexpr int value = 3; };
template <> struct GradMinBlocks<double> { static constexpr int value = 1; };

template <typename T, bool ANCH>
__global__ void __launch_bounds__(kWarpsPerBlock * kWarp, GradMinBlocks<T>::value)
pairhmm_grad_kernel(const BatchView bv, const GradView gv, const Tables<T>* __restrict__ gtab,
                    const Scalars<T> sc, const GradTables* __restrict__ gtt, const GradScalars gs) {
  __shared__ Tables<T> tab;
  __shared__ GradTables gt;
  {
    const int words = (int)(sizeof(Tables<T>) / sizeof(int));
    const int* src = reinterpret_cast<const int*>(gtab);
    int* dst = reinterpret_cast<int*>(&tab);
    for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    const int gwords = (int)(sizeof(GradTables) / sizeof(int));
    const int* gsrc = reinterpret_cast<const int*>(gtt);
    int* gdst = reinterpret_cast<int*>(&gt);
    for (int i = threadIdx.x; i < gwords; i += blockDim.x) gdst[i] = gsrc[i];
  }
  __syncthreads();
  extern __shared__ __align__(16) unsigned char grad_dyn[];
  const int lane = threadIdx.x & (kWarp - 1);
  const long long gw = (long long)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  T* slot = reinterpret_cast<T*>(gv.scratch + gw * gv.slot_bytes);
  T* sbuf = reinterpret_cast<T*>(grad_dyn + (threadIdx.x >> 5) * grad_smem_per_warp<T>());
  long long total = gv.n_items;
  if (gv.count != nullptr) {
    const long long c = (long long)*gv.count;
    total = c < total ? c : total;
  }
  for (;;) {
    unsigned long long i = 0;
    if (lane == 0) i = atomicAdd(gv.head, 1ull);
    i = __shfl_sync(0xffffffffu, i, 0);
    if ((long long)i >= total) break;
    const RescueEntry item = gv.items[i];
    const int code = bv.read_code[item.read];
    const bool gen = code_general(code);
#define VD_GCASE(r)                                                                          \
  case r:                                                                                    \
    if (gen) grad_pair<T, r, true, ANCH>(bv, gv, item, &tab, sc, &gt, gs, lane, slot, sbuf); \
    else grad_pair<T, r, false, ANCH>(bv, gv, item, &tab, sc, &gt, gs, lane, slot, sbuf);    \
    break;
    switch (code_R(code)) {
      VD_GCASE(1) VD_GCASE(2) VD_GCASE(3) VD_GCASE(4) VD_GCASE(5) VD_GCASE(6) VD_GCASE(7) VD_GCASE(8)
      default: break;
    }
#undef VD_GCASE
  }
}

}  // namespace vd
