/*
 * vardepth_pairhmm.h — C ABI of the B200 (sm_100a) PairHMM read x haplotype
 * likelihood stage.  Link against libvardepth_pairhmm.so.
 *
 * Results are natural-log likelihoods (float64), like every reference entry
 * point; an empty read or haplotype gives -inf.  Status codes follow the
 * reference's C ABI (caller/native/caller/batch_hmm.cpp:192-199,
 * trie_vector.cpp:284-286): 0 = OK, 1 = bad arguments; codes >= 2 are device
 * errors this library adds.  vd_last_error() describes the last failure of
 * the calling thread.  All inputs are caller-owned host memory (device memory
 * for vd_forward_region_noalloc); nothing is retained after a call returns
 * (plans excepted, see below).
 */
#ifndef VARDEPTH_PAIRHMM_H
#define VARDEPTH_PAIRHMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  VD_OK = 0,
  VD_EINVAL = 1,   /* bad arguments (same meaning as the reference's return 1) */
  VD_ECUDA = 2,    /* CUDA runtime error */
  VD_ENODEV = 3,   /* no usable CUDA device */
  VD_ENOMEM = 4,   /* device or host allocation failed, or a pair exceeds the budget */
  VD_EOVERFLOW = 5 /* a rescue list overflowed (internal capacity error) */
};

enum {
  VD_PRECISION_MIXED = 0,   /* FP32 scaled wavefront, FP64 rescue of underflowing pairs */
  VD_PRECISION_FLOAT64 = 1  /* every pair in the FP64 wavefront */
};

/* How the primary tier assigns pairs to warps. */
enum {
  VD_SCHEDULE_BATCHED = 0,  /* persistent warps on a work queue; one item streams a read through
                               all haplotypes of its region; items grouped by read length (rows
                               per lane) and ordered longest first; two reads per warp where
                               possible */
  VD_SCHEDULE_PLAIN = 1     /* the comparison baseline: one read x haplotype pair per item, a
                               fixed tile of 8 rows per lane (reads longer than one strip keep
                               the engine's strip height), items in input order, assigned
                               round-robin to a fixed grid of warps (no queue, no binning) */
};

/* Model parameters of one call. */
typedef struct vd_params {
  double gap;       /* gap-open probability g (reference production value 0.001) */
  double ext;       /* gap-continuation probability x (reference value 0.1) */
  int anchored;     /* 0: semiglobal (wide.cpp:9-33), 1: anchored/global (anchored.cpp:5-25) */
  int precision;    /* VD_PRECISION_* */
  const double *quality_offsets; /* NULL, or 4 Phred offsets added per quality bin
                                    (bins: q<15, q<25, q<35, q>=35); no counterpart in
                                    the reference, NULL reproduces it exactly */
  int schedule;     /* VD_SCHEDULE_* (0 = batched) */
  int reserved[3];  /* must be zero */
} vd_params;

/* A batch of reads and haplotypes in packed buffers.  Read r occupies
 * read_bases/read_quals[read_off[r] .. read_off[r+1]); haplotype h occupies
 * hap_bases[hap_off[h] .. hap_off[h+1]).  Bases are the reference's bytes
 * (ASCII ACGTN, compared as plain bytes); qualities are Phred bytes 0..255.
 *
 * The pairs to score are given either
 *  - as regions (pair_read == NULL): region g scores every read in
 *    [region_read_off[g], region_read_off[g+1]) against every haplotype in
 *    [region_hap_off[g], region_hap_off[g+1]); the output holds the regions in
 *    order, each a reads x haplotypes row-major block (trie_vector.cpp:284-292
 *    layout, one block per region); or
 *  - as explicit pairs (pair_read != NULL): out[p] scores read pair_read[p]
 *    against haplotype pair_hap[p] (batch_hmm.cpp:192 semantics). */
typedef struct vd_batch {
  const unsigned char *read_bases;
  const unsigned char *read_quals;
  const int64_t *read_off;   /* n_reads + 1 */
  int64_t n_reads;
  const unsigned char *hap_bases;
  const int64_t *hap_off;    /* n_haps + 1 */
  int64_t n_haps;
  const int64_t *region_read_off; /* n_regions + 1 (region form) */
  const int64_t *region_hap_off;  /* n_regions + 1 (region form) */
  int64_t n_regions;
  const int32_t *pair_read;  /* n_pairs (pair form) */
  const int32_t *pair_hap;   /* n_pairs (pair form) */
  int64_t n_pairs;
} vd_batch;

/* Telemetry of one call (the reference's CudaPairHMM.last, accelerator.py:155-158). */
typedef struct vd_stats {
  int64_t pairs;            /* output slots */
  int64_t dp_cells;         /* sum of n*m over non-empty pairs */
  int64_t work_items;       /* warp work items of the primary tier */
  int64_t batches;          /* memory-budget chunks */
  int64_t rescued_fp64;     /* pairs recomputed in the FP64 wavefront */
  int64_t rescued_robust;   /* pairs recomputed in the FP64 32-row-strip tier */
  int64_t h2d_bytes;
  int64_t d2h_bytes;
  int64_t kernel_launches;  /* kernels of this library launched */
  double kernel_ms;         /* device time of the DP kernels (CUDA events) */
  double total_ms;          /* host wall time of the call */
  double host_ms;           /* host packing time */
  int64_t live_bytes;       /* device bytes held by the call's buffers */
  double primary_ms;        /* device time of the primary (FP32, or FP64) tier alone */
  double rescue_ms;         /* device time of the two FP64 rescue tiers */
  int64_t shared_cells;     /* of dp_cells, those of haplotype columns that repeat the previous
                               haplotype of the region and were not streamed again */
  int64_t rescued_fp32;     /* pairs the primary tier spilled that the FP32 drift tier (per-row
                               power-of-two boosts, semiglobal) resolved */
  int64_t long_strips;      /* strips of the long-read warp kernel (per pair of an item) */
  int64_t long_strip_runs;  /* their runs: a strip whose bottom left the window runs again */
} vd_stats;

typedef struct vd_engine vd_engine;
typedef struct vd_plan vd_plan;

/* ---- engine --------------------------------------------------------------
 * One engine per device and process (accelerator.py:80-103 CudaPairHMM).  It
 * owns a stream, cached device buffers and per-parameter tables.  memory_mb
 * bounds the device bytes of one batch; larger inputs run as several batches
 * (accelerator.py:118-121).  Calls on one engine are serialised. */
int vd_engine_create(int device, int64_t memory_mb, vd_engine **out);
int vd_engine_destroy(vd_engine *engine);
/* Name of the device, compute capability and SM count. */
int vd_engine_info(const vd_engine *engine, char *name, int name_len, int *major, int *minor,
                   int *sm_count);

/* Work-list choices of an engine, applied to the batches it builds from then
 * on (the autotuner in vardepth_b200/autotune.py measures and sets them).
 * No counterpart in the reference. */
typedef struct vd_tuning {
  int long_read_rows;   /* strip height of reads longer than 256 bases: 64, 128 or 256 (default;
                           VD_LONG_WARP runs 128 or 256);
                           shorter strips are renormalised more often, so error-rich long reads
                           stay in the FP32 tier */
  int pair_mask;        /* bit R (1..8): two reads with R rows per lane may share a warp in the
                           packed FP32 kernel (default 0x1fe: every R) */
  int max_item_columns; /* haplotype columns one work item streams at most; 0 = unlimited (default) */
  int pipeline_gcells;  /* vd_forward cuts a batch of N >= 2 x this many 1e9 DP cells into
                           min(8, N / this) chunks (the first a quarter of the others), so the
                           host work and copies of one chunk overlap the kernels of the previous
                           one; 0 = the default (300), 1e6 or more = one chunk */
  int long_mode;        /* reads longer than one strip, FP32 semiglobal: VD_LONG_WARP (default) runs a
                           read against two haplotypes per warp with per-lane power-of-two boosts;
                           VD_LONG_BLOCK the same items on a block per item, whose 4 warps split
                           each strip (4x shorter latency per pair, for batches of few long
                           pairs); VD_LONG_SINGLE the single-read kernel (strips renormalised
                           exactly, error-rich reads then rescued by the drift tier) */
  int pair_split;       /* two-read items with at least this many rows per lane (6, the default, or 7)
                           run on the 12-warp-per-SM kernel (168 registers), fewer rows on the
                           16-warp kernel (128 registers); 0 = 6 */
  int long_group;       /* VD_LONG_WARP: haplotypes per long-read item, 1..8 (0 = 8).  The item's
                           warp runs them two at a time; the pairs after the first take each
                           strip's lane boosts from the first pair's measured decays (the read's
                           errors sit at the same rows against every haplotype), so fewer strips
                           run twice.  Fewer haplotypes per item leave more items for a batch
                           of few long reads.  VD_LONG_BLOCK items hold two haplotypes. */
  int reserved[1];      /* must be zero */
} vd_tuning;
enum { VD_LONG_WARP = 0, VD_LONG_SINGLE = 1, VD_LONG_BLOCK = 2 };
int vd_engine_set_tuning(vd_engine *engine, const vd_tuning *tuning);
int vd_engine_get_tuning(const vd_engine *engine, vd_tuning *tuning);

/* Score a batch (host buffers in, host out).  Replaces CudaPairHMM.score
 * (accelerator.py:105-159): packing, transfers, the kernels and the FP64
 * rescue all happen here.  out must hold vd_batch_outputs(batch) doubles. */
int vd_forward(vd_engine *engine, const vd_batch *batch, const vd_params *params, double *out,
               vd_stats *stats);
int64_t vd_batch_outputs(const vd_batch *batch);

/* The order and shared prefixes in which the two-read kernels stream one
 * region's haplotypes (no counterpart in the reference: it exposes the rule of
 * the work-list build, which runs on the host and needs no device).  order[i]
 * is the haplotype (0 .. n_haps-1) at position i: lexicographic order of the
 * bases, shorter first on a common prefix, ties in input order.  share[i] = Q
 * >= 0 when position i starts at DP column Q+1 from the state of column Q
 * that position i-1's stream laid down or started from (the two agree on
 * their first Q bases); -1 when it streams from column 0.  Q < its length and
 * Q >= 32; an empty haplotype shares nothing and ends the chain. */
int vd_prefix_plan(const unsigned char *hap_bases, const int64_t *hap_off, int64_t n_haps, int32_t *order,
                   int32_t *share);

/* ---- plans: device-resident batches --------------------------------------
 * vd_plan_create uploads a batch and builds its work list once (ignoring the
 * memory budget); vd_plan_run replays the kernels (captured once into a CUDA
 * graph) on the resident inputs; vd_plan_fetch copies the results out. */
int vd_plan_create(vd_engine *engine, const vd_batch *batch, const vd_params *params,
                   vd_plan **out);
int vd_plan_run(vd_plan *plan, vd_stats *stats);
int vd_plan_fetch(vd_plan *plan, double *out);
int vd_plan_destroy(vd_plan *plan);

/* ---- drop-ins for the reference's CPU entry points -----------------------
 * Same arguments and results as the reference functions named, computed on
 * the default engine (device VARDEPTH_CUDA_DEVICE, default 0).  The constant
 * gap 0.001 / ext 0.1 of the batch kernels is kept where the reference
 * hard-codes it. */

/* caller/native/caller/batch_hmm.cpp:192 pairhmm_pairs: count independent pairs,
 * mode 0/2 semiglobal, 1 anchored; lanes is accepted and ignored. */
int vd_pairhmm_pairs(const char *const *reads, const unsigned char *const *quals, const int *rn,
                     const char *const *haps, const int *hn, int count, int mode, int lanes,
                     double *out);
/* caller/native/caller/trie_vector.cpp:284 trie_many: nr reads x nh haplotypes,
 * out row-major by read; *cells receives the DP cells computed. */
int vd_trie_many(const char *const *reads, const unsigned char *const *quals, const int *rn, int nr,
                 const char *const *haps, const int *hn, int nh, int mode, int lanes, double *out,
                 uint64_t *cells);
/* caller/native/caller/wide.cpp:349 read_haplotype_batch_mode: one read x count
 * haplotypes with explicit gap/ext (void in the reference; status here). */
int vd_read_haplotype_batch_mode(const char *read, const unsigned char *qual, int n,
                                 const char *const *haps, const int *lengths, int count, double gap,
                                 double ext, double *out, int mode);
/* caller/native/caller/wide.cpp:9 read_haplotype and anchored.cpp:5 anchored_pairhmm:
 * one pair (NaN on a device error). */
double vd_read_haplotype(const char *read, const unsigned char *qual, int n, const char *hap, int m,
                         double gap, double ext);
double vd_anchored_pairhmm(const char *read, const unsigned char *qual, int n, const char *hap,
                           int m, double gap, double ext);

/* ---- the Python pair-list drop-in -----------------------------------------
 * caller/native/caller/accelerator.py:166-186 score_pairs and :105-159
 * CudaPairHMM.score take a list of (read, qualities, haplotype) triples; the
 * Python layer of this library hands it over as the pointer arrays of the
 * batch_hmm.cpp:192 convention (read, quality and haplotype pointers, read and
 * haplotype lengths, one entry per pair), and this call does the rest of the
 * host work natively: every distinct read and haplotype is checked for
 * uppercase ACGTN (VD_EINVAL, "Uppercase DNA required", accelerator.py:31-33),
 * identical reads (bases and qualities) and haplotypes are stored once,
 * repeated pairs are scored once, and reads that ask for the same set of
 * haplotypes are regrouped into one region, so the batch reaches the packed
 * two-read kernels and the shared-prefix schedule.  out[p] (count doubles)
 * receives pair p's ln L; empty reads or haplotypes give -inf.  The pointers
 * are only read during the call. */
int vd_score_pair_list(vd_engine *engine, const char *const *reads, const unsigned char *const *quals,
                       const int *rn, const char *const *haps, const int *hn, int64_t count,
                       const vd_params *params, double *out, vd_stats *stats);
/* The regrouping vd_score_pair_list applies, on the host only (no device is
 * used; no counterpart in the reference).  counts[4] receives the distinct
 * reads, distinct haplotypes, regions and output slots of the region batch;
 * the nullable per-pair arrays receive the distinct read id, haplotype id
 * (both in order of first appearance), region (regions in order of their
 * first read) and the pair's slot in the region batch's output (regions in
 * order, each a reads x haplotypes row-major block, haplotypes in id order). */
int vd_pair_list_plan(const char *const *reads, const unsigned char *const *quals, const int *rn,
                      const char *const *haps, const int *hn, int64_t count, int64_t *counts,
                      int32_t *pair_read, int32_t *pair_hap, int32_t *pair_region, int64_t *pair_slot);

/* ---- gradient --------------------------------------------------------------
 * No counterpart in the reference (it has no differentiable PairHMM).  For the
 * semiglobal model, every pair's ln L and its six partial derivatives
 *   jac[6 o + k] = d ln L_o / d theta_k,
 *   theta = (Qg, Qx, o0, o1, o2, o3):  gap = 10^(-Qg/10), ext = 10^(-Qx/10),
 *   and o_b the Phred offset of quality bin b (the bins of vd_params), so
 *   that the error of a base with Phred q in bin b is 10^(-max(0, min(q,60) + o_b)/10).
 * The derivatives are taken at params (gap, ext, quality_offsets; NULL offsets
 * = all 0) by a reverse-wavefront sweep over the DP (reverse-mode
 * differentiation of the scaled forward recurrence): FP32 for every pair
 * whose FP32 forward stays in range, FP64 for the rest (all pairs with
 * precision = VD_PRECISION_FLOAT64).  Memory: VD_CHECKPOINT_SQRT keeps the
 * warp state every ceil(sqrt(T)) anti-diagonals (T = m + 33) and replays one
 * segment at a time; VD_CHECKPOINT_ALL keeps every anti-diagonal.  Both give
 * identical results.  Semiglobal and anchored models; reads of at most 256
 * bases (255 anchored); gap, ext > 0.  In anchored mode the gradient is that of
 * the end cell without the 1e-300 floor of anchored.cpp:24 (which binds only
 * for end cells 1e-300 below the last row's maximum).
 * out_ln and out_jac (6 doubles per output) are host arrays in the output
 * order of vd_forward.  Empty reads or haplotypes give -inf and a zero row. */
enum { VD_CHECKPOINT_SQRT = 0, VD_CHECKPOINT_ALL = 1 };

typedef struct vd_grad_stats {
  int64_t pairs;           /* output slots */
  int64_t dp_cells;        /* sum of n*m over non-empty pairs */
  int64_t fp64_pairs;      /* pairs differentiated in the FP64 pass */
  int64_t failed_pairs;    /* NaN results: the FP64 pass underflowed as well */
  int64_t scratch_bytes;   /* device bytes of checkpoints and segment buffers */
  int64_t kernel_launches;
  double kernel_ms;        /* device time of the two passes (CUDA events) */
  double total_ms;         /* host wall time of the call */
} vd_grad_stats;

int vd_forward_backward(vd_engine *engine, const vd_batch *batch, const vd_params *params, int checkpoint,
                        double *out_ln, double *out_jac, vd_grad_stats *stats);

/* ---- region genotypes (forward + post-processing on the device) -----------
 * Scores a region batch (region form) and, without copying the likelihoods
 * back, normalises every read's row and sums each region's unordered diploid
 * genotype log-likelihoods, all in FP64 on the device:
 *   v_h = exp(ll_h - max ll), v'_h = (1 - e) v_h + e mean(v), e = 10^(-min(mq,60)/10),
 *   certainty = max_h ln v'_h - min_h ln v'_h  (ln floored at 1e-300)
 *     (caller/native/caller/molecule_rows.py:6-14 normalized_rows);
 *   gl[(a,b)] for b = 0..H-1, a = 0..b (VCF order), over the region's reads:
 *     artifact_prior < 0:  sum ln max(1e-300, (v'_a + v'_b)/2)
 *       (caller/native/caller/triangular.py:13-16);
 *     artifact_prior >= 0: the allele-balance (and, for a prior > 0,
 *       contamination) mixture of caller/native/caller/mixture_general.cpp:9-37.
 * Each read is one molecule (callers that merge mates pass merged rows to the
 * reference's own mixture instead).  mapping_quality: one byte per read, NULL
 * = 60.  out_gl holds sum_g H_g (H_g + 1) / 2 doubles (regions in order);
 * out_ln, out_values (one per output of vd_forward), out_certainty (one per
 * read) and out_guarded (one int per region) may be NULL.
 *
 * Near-tie guard (options->near_tie_guard = 1; the device-side counterpart of
 * caller/native/caller/partial_anchor.py:120-133): a region whose best two
 * genotypes lie within 1e-4 x max(1, reads) of each other, by GL or by GL
 * plus the uniform haplotype prior (1 for a == b, 2 otherwise), is flagged on
 * the device and rescored in FP64 (VD_PRECISION_FLOAT64, within 2e-9 of the
 * reference's CPU FP64), so its genotype call follows the FP64 convention;
 * out_guarded[g] = 1 marks those regions.  No counterpart in the reference as
 * one call. */
typedef struct vd_genotype_options {
  double artifact_prior;  /* < 0: no artifact prior; >= 0: the mixtures above */
  int near_tie_guard;     /* 1: rescore near-tied regions in FP64 */
  int reserved[3];        /* must be zero */
} vd_genotype_options;

int vd_region_genotypes(vd_engine *engine, const vd_batch *batch, const vd_params *params,
                        const unsigned char *mapping_quality, const vd_genotype_options *options,
                        double *out_ln, double *out_values, double *out_certainty, double *out_gl,
                        int *out_guarded, vd_stats *stats);

/* ---- a call that allocates nothing ----------------------------------------
 * No counterpart in the reference.  For callers that may not call cudaMalloc
 * or any allocating routine: code running under a framework's caching
 * allocator or a fixed memory pool that must not be bypassed, processes that
 * forbid driver allocations after start-up, and code that must not block on
 * the allocator.  Scores one region -- every read against every haplotype,
 * out[r * n_haps + h] -- whose inputs (packed as in vd_batch) and output the
 * caller holds in DEVICE memory of `device`, enqueued on `stream` (a
 * cudaStream_t; NULL = the legacy default stream), and waits for that stream
 * before returning.
 *
 * All scratch (counters, work codes, rescue lists, strip boundaries, model
 * tables) is one fixed static device array of about 8 MiB, which every GPU that
 * loads this library holds until the process exits.  Limits per call: at most
 * 131072 reads, 4096 haplotypes and 131072 read x haplotype pairs, reads of at
 * most 255 bases and haplotypes of at most 1023 bases; larger regions are
 * rejected with VD_EINVAL (split them).  The first call on a device looks up
 * the array's device address and the grid sizes, so make that first call
 * before any stream capture.  Every call shares the one array (the previous
 * call's contents stay in it; each call clears what must start at zero), so
 * overlapping calls on one device would race on it and must not happen; calls
 * from several host threads on the same device are serialised by a per-device
 * lock.  Every buffer must be device (or managed) memory of `device`, checked
 * with cudaPointerGetAttributes before anything is enqueued (VD_EINVAL
 * otherwise). */
int vd_forward_region_noalloc(int device, const unsigned char *read_bases,
                              const unsigned char *read_quals, const int64_t *read_off,
                              int64_t n_reads, const unsigned char *hap_bases,
                              const int64_t *hap_off, int64_t n_haps, const vd_params *params,
                              double *out, void *stream);

/* ---- misc ---------------------------------------------------------------- */
const char *vd_last_error(void);
/* FP32 FMA throughput of a device in TFLOP/s (2 flops per FMA), measured with
 * a register-resident FMA loop: the denominator of the FP32-pipe roofline. */
int vd_measure_fp32_peak(int device, double *tflops);
int vd_device_count(void);
const char *vd_version(void);

#ifdef __cplusplus
}
#endif

#endif /* VARDEPTH_PAIRHMM_H */
