/*
 * kestrel_gpu.h — C ABI of the B200 all-pairs maximum-likelihood Jacquard
 * estimator (libkestrel_gpu.so).
 *
 * This is the drop-in boundary for the path the reference (malariagen/kestrel
 * v0.1.2, Rust) runs from its CLI and Python module:
 *   src/wrapper.rs:89-96   calculate_relatedness_coefficients_gl(...)
 *   src/wrapper.rs:22-29   calculate_relatedness_coefficients_gt(...)
 *   src/coefficients.rs:40-141  the per-pair SQP driver they call
 *   src/coefficients.rs:143-151 struct Output
 * Every entry point takes plain pointers and sizes, returns a kg_status, and
 * never lets a C++ exception or a CUDA error escape; kg_last_error() gives the
 * message of the calling thread's last failing call.  Buffers are caller-owned.  One context per host thread, except the
 * serving calls (kg_panel_*, kg_submit/kg_poll/kg_wait/kg_cancel), which are
 * thread-safe.
 *
 * Genotype codes are the reference's unphased triangular index
 * (src/coefficients.rs:19-38): 0 = 0/0, 1 = 0/1, 2 = 1/1; KG_MISSING (3) marks
 * a missing call, which the reference turns into a NaN likelihood row
 * (src/vcf.rs:397) and drops for that pair only (src/lanevector.rs:99-104).
 * Codes are sample-major: codes[sample * row_stride + site].
 *
 * A call that estimates whole cohorts runs all its waves inside one CUDA graph
 * launch (a device-side loop).  Kernel profilers cannot see kernels inside such
 * graphs; with the environment variable KESTREL_HOST_WAVES=1 the host drives
 * every wave instead (same results, one graph launch per wave).
 */
#ifndef KESTREL_GPU_H
#define KESTREL_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KG_MISSING 3

/* One estimated pair; the reference's Output (src/coefficients.rs:143-151).
 * jacquard[0..8] = Delta1..Delta9; cond is the raw condition estimate (the CLI
 * prints log10(cond), src/cli.rs:170); cond = NaN when the SQP ran out of
 * iterations (src/sqp.rs:92). */
typedef struct {
    uint64_t x;
    uint64_t y;
    double jacquard[9];
    double obj;
    uint64_t iters;
    double cond;
} kg_output;

typedef enum {
    KG_OK = 0,
    KG_EINVAL = 1,      /* bad argument (the reference panics/asserts here) */
    KG_ENOMEM = 2,      /* device or host allocation failed / over budget */
    KG_ECUDA = 3,       /* CUDA runtime or kernel error */
    KG_ETIMEOUT = 4,    /* kg_wait timed out, or a bounded device wait gave up */
    KG_ENOSITES = 5,    /* no segregating site, or a pair with no jointly
                           observed site (the reference asserts,
                           src/lanevector.rs:133-138) */
    KG_ENOTREADY = 6,   /* request still running */
    KG_ENOTFOUND = 7,   /* unknown request id */
    KG_ECANCELED = 8    /* request was cancelled */
} kg_status;

typedef enum {
    KG_PREC_FP32C = 0,  /* FP32 site sums promoted to FP64 every few sites; FP64 solver (default) */
    KG_PREC_FP64 = 1    /* FP64 throughout (the plain FP64 GPU form) */
} kg_precision;

typedef struct kg_ctx kg_ctx;

/* Context on CUDA device `device`.  mem_budget = 0 means no limit beyond the
 * device's free memory. */
int kg_create(kg_ctx **ctx, int device, size_t mem_budget);
int kg_destroy(kg_ctx *ctx);
const char *kg_last_error(const kg_ctx *ctx);
const char *kg_version(void);

/* Arithmetic of the per-site sums (kg_precision). */
int kg_set_precision(kg_ctx *ctx, int precision);

/* Launch shape of the pair engine: pairs in flight per wave (slots; 0 = a
 * fifth of the pairs, from 4096 to 131072, as memory allows) and blocks per SM
 * of the site-pass kernel (0 = the occupancy limit).  Exposed for the
 * autotuner and tests; results do not depend on it. */
int kg_set_launch(kg_ctx *ctx, int slots, int blocks_per_sm);

/* Upper bound on the waves of one call (0 = automatic: a bound from the work
 * that only stops a loop that would not end).  A call that reaches it returns
 * KG_ETIMEOUT with its rows unfinished; the context stays usable and the next
 * call starts afresh.  No counterpart in the reference (its SQP loop is bounded
 * per pair by `iterations`, src/sqp.rs:60); exposed so that the bounded device
 * loop's error path can be exercised without a fault. */
int kg_set_wave_limit(kg_ctx *ctx, uint64_t waves);

/* Pass work unit (the site chunk one warp of the site-pass kernel streams at a
 * time): list entries per unit, a multiple of 512 from 1024 to 65536, or 0 for
 * the default (32768).  It sets how a pass's FP64 partial sums are grouped, so
 * rows can change in their last bits (well inside the parity tolerances).  No
 * counterpart in the reference (its passes stream a pair's rows in 32-row blocks,
 * src/jacquard/grad_hess.rs:10). */
int kg_set_work_unit(kg_ctx *ctx, int entries);

/* The context's launch shape: pairs in flight (0 = automatic), site-pass blocks
 * per SM (0 = occupancy limit), work unit (0 = default) and the divisor of the
 * automatic pairs in flight (the job's pairs / divisor, within 4096..131072).
 * Any pointer may be NULL. */
int kg_get_launch(const kg_ctx *ctx, int *slots, int *blocks_per_sm, int *unit_entries, int *slot_divisor);

/* Runs the autotuner on a sample of the loaded cohort (about 131,072 pairs of
 * its first samples) and keeps the fastest launch shape, by coordinate descent,
 * a change kept only when it is more than 2% faster: site-pass blocks per SM
 * (occupancy limit, 4, 3) and the work unit (32768, 65536, 16384, 8192
 * entries), judged by the site passes' device time; then, for a cohort of
 * fewer than 655,360 pairs, the automatic pairs in flight (a fifth, a third
 * or an eighth of a job's pairs), judged by the sample's whole device time.
 * Writes *slots (0:
 * automatic) and *blocks_per_sm if non-NULL; kg_get_launch reports the rest. */
int kg_autotune(kg_ctx *ctx, int *slots, int *blocks_per_sm);

/* ---------------------------------------------------------------- cohort */

/* Loads a cohort (all n_samples rows feed the allele frequencies). */
int kg_load_genotypes(kg_ctx *ctx, const uint8_t *codes, int64_t n_samples,
                      int64_t n_sites, int64_t row_stride);

/* Same cohort from the host VCF parser's packed form: 2-bit genotype codes,
 * 16 sites per uint32 (site s at bits 2*(s%16) of word s/16, values 0..2), and
 * an observed mask, 32 sites per uint32 (bit s%32 of word s/32 set = called).
 * Rows are ceil(n_sites/16) and ceil(n_sites/32) words long. */
int kg_load_genotypes_2bit(kg_ctx *ctx, const uint32_t *codes2,
                           const uint32_t *observed, int64_t n_samples,
                           int64_t n_sites);

/* Pre-computed allele frequencies, n_sites x 2 ([REF, ALT]) or NULL to estimate
 * them from the samples (the reference's -a estimate). */
int kg_set_allele_frequencies(kg_ctx *ctx, const double *af);

/* Tri- and tetra-allelic sites (the reference's gt3 and gt4 for the CLS
 * estimator, src/coefficients.rs:180-224, and its gl3 / gl4 on one-hot
 * likelihoods for the ML estimator, src/coefficients.rs:99-106):
 * gidx[s * row_stride + v] is sample s's genotype at site v as its index in the
 * VCF order (j (j + 1) / 2 + i for alleles i <= j; 255 = missing), n_alleles[v]
 * the site's allele count (3 or 4), af (n_sites x 4, or NULL) its allele
 * frequencies.  n_samples must be that of the loaded genotypes; loading
 * genotypes again clears these, as does n_sites = 0.
 *   kg_relatedness_gt: a missing call drops the site; frequencies are counts
 *   over all samples unless af is given.
 *   kg_relatedness: a missing call drops the site for that sample's pairs;
 *   frequencies come from the per-site fit over the called samples (capped
 *   at the call's iterations, then the maf cut) unless af is given; alleles
 *   left at zero frequency are dropped (src/wrapper.rs:349-409), a site with
 *   fewer than two left is discarded, and a call that uses a dropped allele
 *   gives its pairs a row of zeros at that site, as the reference's one-hot
 *   likelihoods do. */
int kg_load_multiallelic(kg_ctx *ctx, const uint8_t *gidx, int64_t n_samples, int64_t n_sites,
                         int64_t row_stride, const uint8_t *n_alleles, const double *af);

/* All pairs (x, y), 0 <= x <= y < num_samples, in the reference's row order
 * (outputs[x] then y = x..num_samples-1, src/coefficients.rs:77-136).
 * num_samples < 0 means all samples; iterations is the SQP cap (-i, default
 * 100); maf < 0 or NaN selects 1/(2 n_samples) (src/wrapper.rs:101).
 * out_cap must be >= num_samples*(num_samples+1)/2. */
int kg_relatedness(kg_ctx *ctx, int64_t num_samples, uint64_t iterations,
                   double maf, kg_output *out, int64_t out_cap, int64_t *n_out);

/* The reference's default hard-call estimator (-f GT): conditional least
 * squares with the Brier objective, replacing
 * calculate_relatedness_coefficients_gt (src/wrapper.rs:22-29, the estimator of
 * src/coefficients.rs:166-278).  Only sites that every loaded sample calls are
 * used (the GT reader drops a record with a missing call, src/vcf.rs:217-221);
 * frequencies are the allele counts over all samples (src/wrapper.rs:412-428)
 * or those of kg_set_allele_frequencies, with no maf filter.  Rows as
 * kg_relatedness: obj is the Brier score, iters the QP iterations (at most
 * `iterations`, src/coefficients.rs:207), cond the reduced-Hessian estimate of
 * Q at the solution.  Tri- and tetra-allelic sites of kg_load_multiallelic
 * join Q, c and M.  Returns KG_ENOSITES when no biallelic site is complete. */
int kg_relatedness_gt(kg_ctx *ctx, int64_t num_samples, uint64_t iterations,
                      kg_output *out, int64_t out_cap, int64_t *n_out);

/* The reference's GL/PL estimator on soft genotype likelihoods (src/wrapper.rs:
 * 89-330), biallelic sites: gl is n_samples x n_sites x 3 doubles, sample-major,
 * the linear-scale likelihoods of 0/0, 0/1, 1/1 (the VCF reader's 10^(GL - max)
 * or 10^(-PL/10)); a sample with a NaN at a site is missing there.  Allele
 * frequencies come from the per-site HWE SQP on the likelihoods (capped at
 * `iterations`), with the maf cut (maf < 0 or NaN: 1/(2 n_samples)); each
 * pair's rows are sum over genotype pairs of GLx GLy m(gx, gy), and the SQP is
 * that of kg_relatedness, a warp per pair.  Evaluations follow the context's
 * precision (kg_set_precision): KG_PREC_FP32C evaluates in FP32 from FP32
 * copies of the likelihoods with FP64 sums, and re-runs a pair in FP64 by the
 * rule of kg_relatedness; KG_PREC_FP64 evaluates every pair in FP64.  The
 * device buffers of the call stay with the context for the next call. */
int kg_load_likelihoods(kg_ctx *ctx, const double *gl, int64_t n_samples, int64_t n_sites);
/* Tri- or tetra-allelic sites for kg_relatedness_gl (the reference's gl3 and
 * gl4, src/coefficients.rs:99-106): gl is n_samples x n_sites x G doubles
 * (G = 6 for n_alleles 3, 10 for 4; genotypes in the VCF order, linear scale,
 * a NaN marks a missing sample), n_samples that of kg_load_likelihoods, which
 * clears both classes (as does n_sites = 0).  Their frequencies come from the
 * same per-site fit, then the maf cut and the drop of zero-frequency alleles
 * (src/wrapper.rs:349-409); a pair's row at such a site is the sum over its
 * remaining genotype pairs of GLx GLy m(gx, gy), built once per pair. */
int kg_load_likelihoods_multiallelic(kg_ctx *ctx, const double *gl, int64_t n_samples, int64_t n_sites,
                                     int n_alleles);
int kg_relatedness_gl(kg_ctx *ctx, int64_t num_samples, uint64_t iterations, double maf,
                      kg_output *out, int64_t out_cap, int64_t *n_out);

/* One-shot form of the reference's
 * calculate_relatedness_coefficients_gl(genotype_likelihoods,
 * allele_frequencies, threads, iterations, minimum_allele_frequency,
 * num_samples) (src/wrapper.rs:89-96) on hard calls: creates a context on
 * device 0, loads, runs and destroys it.  `threads` is accepted and ignored
 * (there is no host thread pool on this path). */
int kg_relatedness_coefficients(const uint8_t *codes, int64_t n_samples,
                                int64_t n_sites, int64_t row_stride,
                                const double *allele_frequencies,
                                int64_t threads, uint64_t iterations,
                                double maf, int64_t num_samples,
                                kg_output *out, int64_t out_cap,
                                int64_t *n_out);

/* ------------------------------------------------------------ batching */

/* Several independent cohorts (uneven N, M and missingness) in one persistent
 * launch: each cohort gets its own allele frequencies and all its pairs. */
typedef struct {
    const uint8_t *codes;      /* sample-major, row_stride bytes per row */
    int64_t n_samples;
    int64_t n_sites;
    int64_t row_stride;
    const double *allele_frequencies; /* NULL = estimate */
    int64_t num_samples;       /* < 0 = all */
    kg_output *out;
    int64_t out_cap;
    int64_t n_out;             /* written by the call */
    int32_t status;            /* per-cohort kg_status, written by the call */
} kg_cohort;

int kg_relatedness_batch(kg_ctx *ctx, kg_cohort *cohorts, int n_cohorts,
                         uint64_t iterations, double maf);

/* ------------------------------------------------------------- serving */

/* Serving is continuous batching: worker threads each run a wave engine, and
 * queued requests join a running engine between its waves as memory allows;
 * a request is answered as soon as its own pairs are done. */

/* Makes `codes` the resident reference panel (packed in HBM with its allele
 * frequencies, estimated unless af is given).  Query requests are scored
 * against it until the next kg_panel_load or kg_destroy. */
int kg_panel_load(kg_ctx *ctx, const uint8_t *codes, int64_t n_samples,
                  int64_t n_sites, int64_t row_stride, const double *af,
                  double maf);

/* Queues n_query new samples (codes over the panel's n_sites) for scoring
 * against every panel sample.  site_mask (n_sites bytes, nonzero = use the
 * site) restricts the request to a subset of sites; NULL uses all.  The call
 * copies its inputs and returns at once with a request id. */
int kg_submit(kg_ctx *ctx, const uint8_t *query_codes, int64_t n_query,
              int64_t row_stride, const uint8_t *site_mask,
              uint64_t iterations, int64_t *request_id);

/* *done = 1 once the request has finished (or failed). */
int kg_poll(kg_ctx *ctx, int64_t request_id, int *done);

/* Waits up to timeout_ms (< 0 = forever) and copies the n_query*n_panel rows
 * (x = query index, y = panel index, query-major) to out, then forgets the
 * request.  Returns KG_ETIMEOUT if it is still running. */
int kg_wait(kg_ctx *ctx, int64_t request_id, int64_t timeout_ms,
            kg_output *out, int64_t out_cap, int64_t *n_out);

/* Drops a queued request (a running one finishes but its rows are discarded). */
int kg_cancel(kg_ctx *ctx, int64_t request_id);

/* Serving counters: requests completed, pairs completed, waves run. */
int kg_serving_stats(kg_ctx *ctx, int64_t *requests, int64_t *pairs,
                     int64_t *launches);

/* ------------------------------------------------------ no allocation */

/* This entry point has no counterpart in the reference.  It serves callers that
 * cannot allocate device memory (an application that owns every byte through
 * its own pool or reservation, or that must not call the CUDA allocator from
 * this thread): it computes all pairs (x, y), 0 <= x <= y < n_samples, exactly
 * as kg_relatedness does with default settings (FP32C, allele frequencies
 * estimated, maf < 0 or NaN = 1/(2 n_samples)), but calls no cudaMalloc,
 * cudaFree or allocating library routine.
 *   d_codes: device pointer to the genotype codes (sample-major, row_stride
 *            bytes per sample, 0/1/2, 3 = missing);
 *   d_out:   device pointer to out_cap >= n_samples*(n_samples+1)/2 rows;
 *   stream:  a cudaStream_t (NULL = the default stream); the call is
 *            synchronous: it waits on that stream and returns once the rows
 *            are written.
 * Limits: n_samples <= 512 and n_sites <= 32768; larger inputs return
 * KG_ENOMEM.  Every intermediate lives in one 48 MiB file-scope __device__
 * array that each GPU loading the library holds until the process exits.  Its
 * device address is looked up on the first call on each device, so make that
 * first call before any stream capture; the address is kept for the life of
 * the process, so do not use this entry point across a cudaDeviceReset.  All
 * calls share the array: calls that overlap on the GPU (other host threads,
 * other streams) race and must be serialised by the caller.  A CUDA error the
 * calling thread left pending makes the call return KG_ECUDA at once and is
 * left pending. */
int kg_relatedness_noalloc(const uint8_t *d_codes, int64_t n_samples,
                           int64_t n_sites, int64_t row_stride,
                           uint64_t iterations, double maf, kg_output *d_out,
                           int64_t out_cap, void *stream);

/* --------------------------------------------------------- diagnostics */

/* Per-run counters of the last kg_relatedness / batch call: grad-Hessian and
 * objective site passes (summed over pairs), pairs that escalated to FP64,
 * kernel launches, and the device time of the pair kernel in milliseconds. */
typedef struct {
    uint64_t gh_passes;
    uint64_t obj_passes;
    uint64_t fp64_passes;
    uint64_t fp64_pairs;
    uint64_t pair_sites;       /* sum over pairs of jointly observed sites */
    uint64_t work_units;       /* sum over passes of sites visited */
    uint64_t launches;         /* kernels launched by the call */
    uint64_t flops_fp32;       /* executed FP32 site arithmetic (FMA = 2) */
    uint64_t flops_fp64;       /* executed FP64 site arithmetic */
    uint64_t shape_sites[5];   /* pair-sites per genotype-pair shape A,B1,B2,C,D */
    uint64_t nonconverged;     /* pairs that stopped at the iteration limit */
    uint64_t waves;            /* admit / pass / solve waves of the pair engine */
    uint64_t slots;            /* pairs in flight per wave */
    double admit_ms;           /* CUDA-event time of the admit kernels (list build) */
    double pass_ms;            /* CUDA-event time of the site-pass kernels */
    double solve_ms;           /* CUDA-event time of the solve kernels (SQP steps) */
    double pair_kernel_ms;     /* CUDA-event time of all pair-engine waves */
    double device_ms;          /* CUDA-event time of preparation + pair kernel */
    double total_ms;           /* host time of the call */
    uint64_t sites_used[3];    /* sites the estimate used, by the alleles they keep (2, 3, 4) after the
                                  frequency cut and the drop of zero-frequency alleles: the reference's
                                  "Identified N di-/tri-/tetra-allelic sites" (src/wrapper.rs:321-323) */
    uint64_t sites_discarded;  /* loaded sites left out (fewer than two alleles left, or for the CLS
                                  estimator a missing call) */
} kg_run_stats;

int kg_last_run_stats(kg_ctx *ctx, kg_run_stats *stats);

/* Measured FP32 FMA throughput of `device` (TFLOP/s, FMA = 2 FLOP) from a
 * register-resident FFMA loop over every SM; the roofline denominator of the
 * FP32 pair kernel. */
int kg_fp32_peak(int device, double *tflops);

/* Runs the reference-compatible CLI (`kestrel input.vcf kinship.tsv [flags]`,
 * src/cli.rs:12-127) in-process; argv[0] is the program name. */
int kg_run_cli(int argc, const char *const *argv);

/* ------------------------------------------------------------ VCF reader */

/* The VCF reader the CLI uses, replacing the reference's parse_vcf with the GT
 * and GL/PL sample parsers (src/vcf.rs:96-236, :384-421): biallelic SNP
 * records of a plain, gzip or bgzip VCF become genotype codes (0/1/2, 3 =
 * missing).  Records whose REF or ALT is not a single base, or with more than
 * one ALT, are skipped and counted; GL/PL rows reduce to the most likely
 * genotype.  BGZF blocks are inflated and the records parsed on `threads` host
 * threads (<= 0: all).  field is "GT", "GL" or "PL"; af_info != 0 also reads
 * INFO/AF (the reference's -a info).  *out is always set when memory allows;
 * on failure kg_vcf_error() gives the message (the first bad record in file
 * order).  Free with kg_vcf_free. */
typedef struct kg_vcf kg_vcf;
int kg_vcf_read(const char *path, const char *field, int af_info, int threads, kg_vcf **out);
const char *kg_vcf_error(const kg_vcf *vcf);
/* counts (optional, 7 entries): records, non-SNP records skipped (a base that
 * is not A/C/G/T, or more than four bases), tri- and tetra-allelic records,
 * biallelic GL/PL rows that were not one-hot, SNP records with at least one
 * missing call, and the tri- and the tetra-allelic records kept. */
int kg_vcf_info(const kg_vcf *vcf, int64_t *n_samples, int64_t *n_sites, uint64_t *counts);
/* codes: n_samples x n_sites, sample-major (the layout kg_load_genotypes takes);
 * af: n_sites x 2 [REF, ALT] from INFO/AF (KG_EINVAL if it was not read).
 * Either may be NULL. */
int kg_vcf_codes(const kg_vcf *vcf, uint8_t *codes, double *af);
/* GL/PL files with a likelihood row that is not one-hot (counts[3] > 0): the
 * linear-scale likelihoods, n_samples x n_sites x 3 (sample-major, NaN where
 * missing), the input of kg_load_likelihoods; KG_ENOTFOUND otherwise. */
int kg_vcf_likelihoods(const kg_vcf *vcf, double *gl);
/* The same for the tri- (n_alleles 3, G = 6) or tetra-allelic (4, G = 10)
 * records, in file order: n_samples x (counts[5] or counts[6]) x G, the input
 * of kg_load_likelihoods_multiallelic; KG_ENOTFOUND when every row is one-hot. */
int kg_vcf_likelihoods_multiallelic(const kg_vcf *vcf, int n_alleles, double *gl);
/* The same codes packed as kg_load_genotypes_2bit takes them (2-bit codes and
 * the observed mask, rows of ceil(n_sites/16) and ceil(n_sites/32) words). */
int kg_vcf_codes_2bit(const kg_vcf *vcf, uint32_t *codes2, uint32_t *observed);
/* The tri- and tetra-allelic records (counts[5] + counts[6] of them), the
 * input of kg_load_multiallelic: gidx n_samples x that many genotype indices
 * (sample-major, VCF order; GL/PL rows give their most likely genotype; 255 =
 * a missing call), n_alleles one per record, af (4 per record, KG_EINVAL if
 * INFO/AF was not read).  Any may be NULL.  A GT record with a malformed call
 * after a missing one is left out, as the reference's reader stops at the
 * missing call. */
int kg_vcf_multiallelic(const kg_vcf *vcf, uint8_t *gidx, uint8_t *n_alleles, double *af);
/* Sample name i (NULL when out of range). */
const char *kg_vcf_sample(const kg_vcf *vcf, int64_t i);
void kg_vcf_free(kg_vcf *vcf);

#ifdef __cplusplus
}
#endif

#endif
