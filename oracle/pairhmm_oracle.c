/*
 * ORACLE — test infrastructure only.  Nothing in the vardepth_b200 product path
 * links, loads or calls this file: it is the checker that tests/, the smoke
 * check of __graft_entry__ and the cpu_baseline leg of bench.py compare the
 * CUDA path against.
 *
 * A plain-C FP64 (and long double) restatement of VarDepth's 3-state PairHMM
 * forward pass, written from the model's mathematics:
 *
 *   semiglobal (free start/end):   caller/native/caller/wide.cpp:9-33
 *                                   caller/native/caller/base/core/core.cpp:9-30
 *   anchored / global:              caller/native/caller/anchored.cpp:5-25
 *   fixed-constant batch modes 0/1/2: caller/native/caller/batch_hmm.cpp:42-97
 *   error LUT e = 10^(-min(q,60)/10):  caller/native/caller/accelerator.py:23
 *
 * Model (i = read row 1..n, j = haplotype column 1..m, g = gap, x = ext):
 *   E_ij   = read[i-1]==hap[j-1] ? 1-e_i : e_i/3      (plain byte compare)
 *   M[i][j] = E_ij * ((1-2g) M[i-1][j-1] + (1-x) (I[i-1][j-1] + D[i-1][j-1]))
 *   I[i][j] = 0.25 * (g M[i-1][j] + x I[i-1][j])
 *   D[i][j] = g M[i][j-1] + x D[i][j-1]
 *   column 0 (i>=1): M = D = 0, I by the same recurrence
 *   row 0 semiglobal: M = 1/(m+1) for j = 0..m;  anchored: M[0][0] = 1, D[0][j] = g x^(j-1)
 *   Z semiglobal = sum_j (M+I)[n][j];  anchored = (M+I+D)[n][m];  result ln(max(1e-300, Z)) + ln(scales)
 *   n <= 0 or m <= 0 gives -inf.
 *
 * Scaling flavours (they differ only in FP64 rounding):
 *   VDO_ROW_DIVIDE  every row divided by its max (core.cpp, anchored.cpp, batch mode 0/1)
 *   VDO_POW2        rows multiplied by 2^512 once their max falls under 2^-450 (wide.cpp, batch mode 2)
 *
 * The quality-offset extension (per-quality-bin Phred offsets, used by the
 * differentiable path) has no counterpart in the reference: with every offset 0
 * it reduces exactly to the reference's error LUT.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <unistd.h>

enum { VDO_ROW_DIVIDE = 0, VDO_POW2 = 2 };

static double error_of(unsigned q) {
    unsigned c = q < 60u ? q : 60u;
    return pow(10.0, -(double)c / 10.0);
}

/* Phred of base i after the optional bin offset; bins as documented in
 * vdo_quality_bin. */
int vdo_quality_bin(unsigned q) {
    /* four bins centred on the Q10/Q20/30/40 levels */
    if (q < 15u) return 0;
    if (q < 25u) return 1;
    if (q < 35u) return 2;
    return 3;
}

double vdo_forward_ld_ex(const unsigned char *read, const unsigned char *qual, int n,
                         const unsigned char *hap, int m, double gap, double ext,
                         int anchored, int clamp);

/* Phred of a base after its bin offset is floored at 0 (an error rate of at
 * most 1), as the library's tables do. */
static double error_offset(unsigned q, const double *offsets) {
    if (!offsets) return error_of(q);
    double c = (double)(q < 60u ? q : 60u) + offsets[vdo_quality_bin(q)];
    if (c < 0.0) c = 0.0;
    return pow(10.0, -c / 10.0);
}

double vdo_forward_ex(const unsigned char *read, const unsigned char *qual, int n,
                      const unsigned char *hap, int m, double gap, double ext,
                      int anchored, int scaling, const double *offsets) {
    if (n <= 0 || m <= 0) return -INFINITY;
    size_t w = (size_t)m + 1;
    double *buf = (double *)calloc(6 * w, sizeof(double));
    if (!buf) return NAN;
    double *pm = buf, *pi = buf + w, *pd = buf + 2 * w;
    double *cm = buf + 3 * w, *ci = buf + 4 * w, *cd = buf + 5 * w;
    const double go = 1.0 - 2.0 * gap, gc = 1.0 - ext;
    if (anchored) {
        pm[0] = 1.0;
        for (int j = 1; j <= m; ++j) pd[j] = gap * pow(ext, (double)(j - 1));
    } else {
        for (int j = 0; j <= m; ++j) pm[j] = 1.0 / (double)(m + 1);
    }
    double log_scale = 0.0;
    for (int i = 1; i <= n; ++i) {
        const double e = error_offset(qual[i - 1], offsets);
        const double hit = 1.0 - e, miss = e / 3.0;
        const unsigned char b = read[i - 1];
        cm[0] = 0.0; cd[0] = 0.0;
        ci[0] = 0.25 * (gap * pm[0] + ext * pi[0]);
        double top = ci[0];
        for (int j = 1; j <= m; ++j) {
            const double emit = (b == hap[j - 1]) ? hit : miss;
            cm[j] = emit * (go * pm[j - 1] + gc * (pi[j - 1] + pd[j - 1]));
            ci[j] = 0.25 * (gap * pm[j] + ext * pi[j]);
            cd[j] = gap * cm[j - 1] + ext * cd[j - 1];
            const double s = cm[j] + ci[j] + cd[j];
            if (s > top) top = s;
        }
        if (!(top > 0.0)) { free(buf); return -INFINITY; }
        if (anchored || scaling == VDO_ROW_DIVIDE) {
            for (int j = 0; j <= m; ++j) { cm[j] /= top; ci[j] /= top; cd[j] /= top; }
            log_scale += log(top);
        } else if (top < 0x1p-450) {
            for (int j = 0; j <= m; ++j) { cm[j] *= 0x1p512; ci[j] *= 0x1p512; cd[j] *= 0x1p512; }
            log_scale -= 512.0 * log(2.0);
        }
        double *t;
        t = pm; pm = cm; cm = t;
        t = pi; pi = ci; ci = t;
        t = pd; pd = cd; cd = t;
    }
    double z = 0.0;
    if (anchored) z = pm[m] + pi[m] + pd[m];
    else for (int j = 0; j <= m; ++j) z += pm[j] + pi[j];
    free(buf);
    return log(z > 1e-300 ? z : 1e-300) + log_scale;
}

double vdo_forward(const unsigned char *read, const unsigned char *qual, int n,
                   const unsigned char *hap, int m, double gap, double ext,
                   int anchored, int scaling) {
    return vdo_forward_ex(read, qual, n, hap, m, gap, ext, anchored, scaling, NULL);
}

/* Extended-precision variant (x87 long double, 64-bit mantissa, exponent
 * range to 2^-16382), renormalised only by exact powers of two: an
 * independent check on the rescaled FP64 arithmetic, free of its underflow.
 * clamp = 1 applies the reference's anchored 1e-300 floor (see below). */
double vdo_forward_ld_ex(const unsigned char *read, const unsigned char *qual, int n,
                         const unsigned char *hap, int m, double gap, double ext,
                         int anchored, int clamp) {
    if (n <= 0 || m <= 0) return -INFINITY;
    size_t w = (size_t)m + 1;
    long double *buf = (long double *)calloc(6 * w, sizeof(long double));
    if (!buf) return NAN;
    long double *pm = buf, *pi = buf + w, *pd = buf + 2 * w;
    long double *cm = buf + 3 * w, *ci = buf + 4 * w, *cd = buf + 5 * w;
    const long double G = gap, X = ext, go = 1.0L - 2.0L * G, gc = 1.0L - X;
    if (anchored) {
        pm[0] = 1.0L;
        long double d = G;
        for (int j = 1; j <= m; ++j) { pd[j] = d; d *= X; }
    } else {
        for (int j = 0; j <= m; ++j) pm[j] = 1.0L / (long double)(m + 1);
    }
    long double log_scale = 0.0L;
    for (int i = 1; i <= n; ++i) {
        unsigned q = qual[i - 1] < 60 ? qual[i - 1] : 60;
        const long double e = powl(10.0L, -(long double)q / 10.0L);
        const long double hit = 1.0L - e, miss = e / 3.0L;
        const unsigned char b = read[i - 1];
        cm[0] = 0.0L; cd[0] = 0.0L;
        ci[0] = 0.25L * (G * pm[0] + X * pi[0]);
        long double top = ci[0];
        for (int j = 1; j <= m; ++j) {
            const long double emit = (b == hap[j - 1]) ? hit : miss;
            cm[j] = emit * (go * pm[j - 1] + gc * (pi[j - 1] + pd[j - 1]));
            ci[j] = 0.25L * (G * pm[j] + X * pi[j]);
            cd[j] = G * cm[j - 1] + X * cd[j - 1];
            long double s = cm[j] + ci[j] + cd[j];
            if (s > top) top = s;
        }
        if (!(top > 0.0L)) { free(buf); return -INFINITY; }
        /* exact power-of-two renormalisation keeps the long double path free of
         * division rounding */
        int ex;
        frexpl(top, &ex);
        if (ex < -4000) {
            for (int j = 0; j <= m; ++j) { cm[j] = ldexpl(cm[j], -ex); ci[j] = ldexpl(ci[j], -ex); cd[j] = ldexpl(cd[j], -ex); }
            log_scale += (long double)ex * logl(2.0L);
        }
        long double *t;
        t = pm; pm = cm; cm = t;
        t = pi; pi = ci; ci = t;
        t = pd; pd = cd; cd = t;
    }
    long double z = 0.0L;
    if (anchored) z = pm[m] + pi[m] + pd[m];
    else for (int j = 0; j <= m; ++j) z += pm[j] + pi[j];
    /* the reference's ln(max(1e-300, Z / S_n)) + ln S_n for the anchored end
     * cell (anchored.cpp:24), with S_n the last row's maximum */
    if (anchored && clamp) {
        long double top = 0.0L;
        for (int j = 0; j <= m; ++j) { long double v = pm[j] + pi[j] + pd[j]; if (v > top) top = v; }
        if (z < 1e-300L * top) z = 1e-300L * top;
    }
    free(buf);
    if (!(z > 0.0L)) return -INFINITY;
    return (double)(logl(z) + log_scale);
}

double vdo_forward_ld(const unsigned char *read, const unsigned char *qual, int n,
                      const unsigned char *hap, int m, double gap, double ext, int anchored) {
    return vdo_forward_ld_ex(read, qual, n, hap, m, gap, ext, anchored, 1);
}

/* Batch over explicit (read, haplotype) pairs held in packed buffers:
 * read r occupies bases/quals[read_off[r] .. read_off[r+1]), haplotype h
 * occupies haps[hap_off[h] .. hap_off[h+1]).  threads <= 0 uses every online
 * core; pairs are handed out in blocks of 16 through an atomic counter. */
typedef struct {
    const unsigned char *bases, *quals, *haps;
    const int64_t *read_off, *hap_off;
    const int32_t *pair_read, *pair_hap;
    int64_t count, next;
    double gap, ext;
    int anchored, scaling, precision_ld;
    double *out;
} vdo_job;

static void *vdo_worker(void *arg) {
    vdo_job *job = (vdo_job *)arg;
    for (;;) {
        int64_t begin = __atomic_fetch_add(&job->next, 16, __ATOMIC_RELAXED);
        if (begin >= job->count) break;
        int64_t end = begin + 16 < job->count ? begin + 16 : job->count;
        for (int64_t p = begin; p < end; ++p) {
            int32_t r = job->pair_read[p], h = job->pair_hap[p];
            const unsigned char *rd = job->bases + job->read_off[r];
            const unsigned char *ql = job->quals + job->read_off[r];
            int n = (int)(job->read_off[r + 1] - job->read_off[r]);
            const unsigned char *hp = job->haps + job->hap_off[h];
            int m = (int)(job->hap_off[h + 1] - job->hap_off[h]);
            job->out[p] = job->precision_ld
                ? vdo_forward_ld(rd, ql, n, hp, m, job->gap, job->ext, job->anchored)
                : vdo_forward(rd, ql, n, hp, m, job->gap, job->ext, job->anchored, job->scaling);
        }
    }
    return NULL;
}

int vdo_forward_pairs(const unsigned char *bases, const unsigned char *quals,
                      const int64_t *read_off, const unsigned char *haps,
                      const int64_t *hap_off, const int32_t *pair_read,
                      const int32_t *pair_hap, int64_t count, double gap, double ext,
                      int anchored, int scaling, int precision_ld, int threads,
                      double *out) {
    if (count < 0 || (count > 0 && !out)) return 1;
    vdo_job job = {bases, quals, haps, read_off, hap_off, pair_read, pair_hap,
                   count, 0, gap, ext, anchored, scaling, precision_ld, out};
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    int started = 0;
    for (int t = 1; t < threads; ++t)
        if (pthread_create(&tid[started], NULL, vdo_worker, &job) == 0) ++started;
    vdo_worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    return 0;
}

/* ---- gradient oracle --------------------------------------------------------
 * d ln L / d theta for theta = (gap-open Phred Qg, gap-continuation Phred Qx,
 * quality-bin offsets o0..o3), g = 10^(-Qg/10), x = 10^(-Qx/10),
 * e_i = 10^(-max(0, min(q_i,60) + o_bin(q_i))/10).  The reference has no
 * differentiable PairHMM; this is the forward-backward (expected-count)
 * gradient of the model of wide.cpp:9-33 / anchored.cpp:5-25 in x87 long
 * double without rescaling (exponent range to 2^-16382), for small cases:
 *
 *   alpha = the forward DP of vdo_forward_ex, beta = dZ/d(cell) (the adjoint
 *   of every cell, accumulated in reverse topological order), and
 *   dZ/dg = sum beta_M E (-2) M[i-1][j-1] + beta_I M[i-1][j]/4 + beta_D M[i][j-1]
 *   dZ/dx = sum beta_M E (-1)(I+D)[i-1][j-1] + beta_I I[i-1][j]/4 + beta_D D[i][j-1]
 *   dZ/de_i = sum_j beta_M[i][j] M[i][j] (match ? -1/(1-e) : 1/e)
 *
 * i.e. the expected transition counts times d ln(transition)/d theta.  The
 * anchored 1e-300 floor of anchored.cpp:24 is not differentiated (where it
 * binds, the value is a constant and its gradient would be 0). */
int vdo_grad_ex(const unsigned char *read, const unsigned char *qual, int n,
                const unsigned char *hap, int m, double gap, double ext, int anchored,
                const double *offsets, double *ln_out, double *jac) {
    for (int k = 0; k < 6; ++k) jac[k] = 0.0;
    if (n <= 0 || m <= 0) { *ln_out = -INFINITY; return 0; }
    const size_t W = (size_t)m + 1, N = ((size_t)n + 1) * W;
    long double *buf = (long double *)calloc(6 * N + 2 * (size_t)n, sizeof(long double));
    if (!buf) return 1;
    long double *FM = buf, *FI = buf + N, *FD = buf + 2 * N;
    long double *BM = buf + 3 * N, *BI = buf + 4 * N, *BD = buf + 5 * N;
    long double *err = buf + 6 * N, *derr = err + n;  /* e_i and de_i / d o */
    const long double G = gap, X = ext, a = 1.0L - 2.0L * G, b = 1.0L - X;
    const long double L10 = logl(10.0L) / 10.0L;
    for (int i = 0; i < n; ++i) {
        unsigned q = qual[i];
        long double ph = (long double)(q < 60u ? q : 60u) + (offsets ? offsets[vdo_quality_bin(q)] : 0.0);
        /* at or below the Phred floor 0 the offset derivative is taken as 0 */
        int clamped = ph <= 0.0L;
        if (clamped) ph = 0.0L;
        err[i] = powl(10.0L, -ph / 10.0L);
        derr[i] = clamped ? 0.0L : -L10 * err[i];
    }
#define IX(i, j) ((size_t)(i) * W + (size_t)(j))
#define EMIT(i, j) ((read[(i) - 1] == hap[(j) - 1]) ? 1.0L - err[(i) - 1] : err[(i) - 1] / 3.0L)
    if (anchored) {
        FM[IX(0, 0)] = 1.0L;
        for (int j = 1; j <= m; ++j) FD[IX(0, j)] = G * FM[IX(0, j - 1)] + X * FD[IX(0, j - 1)];
    } else {
        for (int j = 0; j <= m; ++j) FM[IX(0, j)] = 1.0L / (long double)(m + 1);
    }
    for (int i = 1; i <= n; ++i) {
        FI[IX(i, 0)] = 0.25L * (G * FM[IX(i - 1, 0)] + X * FI[IX(i - 1, 0)]);
        for (int j = 1; j <= m; ++j) {
            FM[IX(i, j)] = EMIT(i, j) * (a * FM[IX(i - 1, j - 1)] + b * (FI[IX(i - 1, j - 1)] + FD[IX(i - 1, j - 1)]));
            FI[IX(i, j)] = 0.25L * (G * FM[IX(i - 1, j)] + X * FI[IX(i - 1, j)]);
            FD[IX(i, j)] = G * FM[IX(i, j - 1)] + X * FD[IX(i, j - 1)];
        }
    }
    long double Z = 0.0L;
    if (anchored) {
        Z = FM[IX(n, m)] + FI[IX(n, m)] + FD[IX(n, m)];
        BM[IX(n, m)] = BI[IX(n, m)] = BD[IX(n, m)] = 1.0L;
    } else {
        for (int j = 0; j <= m; ++j) { Z += FM[IX(n, j)] + FI[IX(n, j)]; BM[IX(n, j)] = 1.0L; BI[IX(n, j)] = 1.0L; }
    }
    if (!(Z > 0.0L)) { free(buf); *ln_out = -INFINITY; return 0; }
    long double dg = 0.0L, dx = 0.0L, dob[4] = {0.0L, 0.0L, 0.0L, 0.0L};
    /* successors of (i,j) are (i+1,j+1), (i+1,j), (i,j+1): reverse row-major
     * order completes every adjoint before it is propagated */
    for (int i = n; i >= 0; --i) {
        long double de = 0.0L;
        for (int j = m; j >= 0; --j) {
            const size_t c = IX(i, j);
            if (i >= 1 && j >= 1) {
                const long double E = EMIT(i, j), bm = BM[c];
                const size_t p = IX(i - 1, j - 1);
                BM[p] += bm * E * a;
                BI[p] += bm * E * b;
                BD[p] += bm * E * b;
                dg += bm * E * (-2.0L) * FM[p];
                dx += bm * E * (-1.0L) * (FI[p] + FD[p]);
                const int match = read[i - 1] == hap[j - 1];
                const long double e = err[i - 1];
                if (derr[i - 1] != 0.0L) de += bm * FM[c] * (match ? -1.0L / (1.0L - e) : 1.0L / e);
            }
            if (i >= 1) {
                const long double bi = BI[c];
                const size_t p = IX(i - 1, j);
                BM[p] += bi * 0.25L * G;
                BI[p] += bi * 0.25L * X;
                dg += bi * 0.25L * FM[p];
                dx += bi * 0.25L * FI[p];
            }
            if (j >= 1 && (i >= 1 || anchored)) {
                const long double bd = BD[c];
                const size_t p = IX(i, j - 1);
                BM[p] += bd * G;
                BD[p] += bd * X;
                dg += bd * FM[p];
                dx += bd * FD[p];
            }
        }
        if (i >= 1) dob[vdo_quality_bin(qual[i - 1])] += de * derr[i - 1];
    }
#undef IX
#undef EMIT
    jac[0] = (double)(dg / Z * (-L10 * G));
    jac[1] = (double)(dx / Z * (-L10 * X));
    for (int k = 0; k < 4; ++k) jac[2 + k] = (double)(dob[k] / Z);
    *ln_out = (double)logl(Z);
    free(buf);
    return 0;
}

typedef struct {
    const unsigned char *bases, *quals, *haps;
    const int64_t *read_off, *hap_off;
    const int32_t *pair_read, *pair_hap;
    int64_t count, next;
    double gap, ext;
    int anchored;
    const double *offsets;
    double *ln, *jac;
    int failed;
} vdo_grad_job;

static void *vdo_grad_worker(void *arg) {
    vdo_grad_job *job = (vdo_grad_job *)arg;
    for (;;) {
        int64_t p = __atomic_fetch_add(&job->next, 1, __ATOMIC_RELAXED);
        if (p >= job->count) break;
        int32_t r = job->pair_read[p], h = job->pair_hap[p];
        int n = (int)(job->read_off[r + 1] - job->read_off[r]);
        int m = (int)(job->hap_off[h + 1] - job->hap_off[h]);
        if (vdo_grad_ex(job->bases + job->read_off[r], job->quals + job->read_off[r], n,
                        job->haps + job->hap_off[h], m, job->gap, job->ext, job->anchored, job->offsets,
                        job->ln + p, job->jac + 6 * p))
            __atomic_store_n(&job->failed, 1, __ATOMIC_RELAXED);
    }
    return NULL;
}

/* vdo_grad_ex over explicit pairs of packed buffers on `threads` host threads. */
int vdo_grad_pairs(const unsigned char *bases, const unsigned char *quals, const int64_t *read_off,
                   const unsigned char *haps, const int64_t *hap_off, const int32_t *pair_read,
                   const int32_t *pair_hap, int64_t count, double gap, double ext, int anchored,
                   const double *offsets, int threads, double *ln, double *jac) {
    if (count < 0 || (count > 0 && (!ln || !jac))) return 1;
    vdo_grad_job job = {bases, quals, haps, read_off, hap_off, pair_read, pair_hap, count, 0,
                        gap, ext, anchored, offsets, ln, jac, 0};
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t tid[256];
    int started = 0;
    for (int t = 1; t < threads; ++t)
        if (pthread_create(&tid[started], NULL, vdo_grad_worker, &job) == 0) ++started;
    vdo_grad_worker(&job);
    for (int t = 0; t < started; ++t) pthread_join(tid[t], NULL);
    return job.failed;
}
