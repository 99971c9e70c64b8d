/*
 * kestrel_oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of the reference's all-pairs maximum-likelihood Jacquard
 * estimator (malariagen/kestrel v0.1.2, the GL/PL path of
 * src/coefficients.rs:40-141 driven by src/wrapper.rs:89-207), applied to hard
 * genotype calls.  It is the checker for the CUDA product path and the timed CPU
 * baseline; nothing in the product links or calls it.
 *
 * Parity status: UNPINNED by the reference itself.  The reference is Rust, no
 * Rust toolchain exists on this machine, and the reference ships no tests, golden
 * vectors or fixtures for this path.  The restatement is pinned instead by
 * independent checks (a numpy evaluation of f, g and H, planted-relationship
 * recovery, the (x,y)/(y,x) swap symmetry and hand-derived small cases).
 *
 * Genotype codes (sample-major, one byte per call):
 *   0 = 0/0, 1 = 0/1, 2 = 1/1   (the reference's unphased triangular index,
 *                               src/coefficients.rs:19-38)
 *   3 = missing call            (the reference's NaN likelihood row,
 *                               src/vcf.rs:397, dropped per pair by
 *                               src/lanevector.rs:99-104)
 */
#ifndef KESTREL_ORACLE_H
#define KESTREL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One row of the reference's output (src/coefficients.rs:143-151). */
typedef struct {
    uint64_t x, y;
    double jacquard[9];
    double obj;
    uint64_t iters;
    double cond;
} kor_output;

enum {
    KOR_OK = 0,
    KOR_EINVAL = 1,
    KOR_ENOMEM = 2,
    KOR_ENOSITES = 5
};

/* Per-site allele counts over observed samples (all n_samples rows). */
int kor_allele_counts(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                      int64_t stride, int32_t *ref_count, int32_t *obs_count);

/* Allele frequencies as the ML path sees them: the reference's GL path on
 * one-hot likelihoods, i.e. the per-site HWE SQP of src/allele/mod.rs:91-134
 * (on the three genotype classes weighted by their counts), maf zeroing
 * (src/allele/mod.rs:120-126), renormalisation, and the non-segregating drop
 * (src/wrapper.rs:366-383).  The SQP's optimum sits about 5e-9 below the count
 * frequency (the eps inside its log), so a count frequency equal to maf is cut.
 * af_in (n_sites x 2, [ref, alt]) overrides the estimate when non-NULL (then
 * only the zero drop applies).  maf < 0 selects the default 1/(2 n_samples). */
int kor_site_frequencies(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                         int64_t stride, const double *af_in, double maf,
                         double *p, double *q, uint8_t *keep, int64_t *n_kept);
/* The same with the allele-frequency SQP's iteration cap (the estimator's
 * `iterations`, src/wrapper.rs:103-131); kor_site_frequencies uses 100. */
int kor_site_frequencies_it(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                            int64_t stride, const double *af_in, double maf, uint64_t iterations,
                            double *p, double *q, uint8_t *keep, int64_t *n_kept);

/* Full all-pairs run for pairs (x, y), 0 <= x <= y < num_samples, in the
 * reference's row order.  num_samples < 0 means all.  threads <= 0 means all
 * OpenMP threads.  out must hold num_samples*(num_samples+1)/2 rows. */
int kor_relatedness(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                    int64_t stride, const double *af_in, int64_t num_samples,
                    uint64_t iterations, double maf, int threads,
                    kor_output *out, int64_t out_cap, int64_t *n_out);

/* The same estimator for an explicit list of pairs, given frequencies already
 * computed by kor_site_frequencies.  Used for sampled parity checks and the
 * bounded CPU baseline. */
int kor_relatedness_pairs(const uint8_t *codes, int64_t n_sites, int64_t stride,
                          const double *p, const double *q, const uint8_t *keep,
                          const int64_t *pair_x, const int64_t *pair_y,
                          int64_t n_pairs, uint64_t iterations, int threads,
                          kor_output *out);

/* f, g, H of one pair at a fixed delta (src/jacquard/objective.rs:9-20,
 * src/jacquard/grad_hess.rs:13-41).  H is 9x9 row-major.  *n_sites_used gets the
 * number of jointly observed segregating sites. */
int kor_eval_pair(const uint8_t *codes_x, const uint8_t *codes_y, int64_t n_sites,
                  const double *p, const double *q, const uint8_t *keep,
                  const double delta[9], double *f, double g[9], double h[81],
                  int64_t *n_sites_used);

/* The reference's default hard-call estimator (-f GT): conditional least
 * squares with the Brier objective (src/coefficients.rs:166-278).  Sites with a
 * missing call in any sample are dropped; frequencies are counts over all
 * samples (or af_in, n_sites x 2); rows as kor_relatedness, with obj = Brier
 * score, iters = QP iterations.  The QP runs at most `iterations` iterations. */
int kor_cls_relatedness(const uint8_t *codes, int64_t n_samples, int64_t n_sites, int64_t stride,
                        const double *af_in, int64_t num_samples, uint64_t iterations, int threads,
                        kor_output *out, int64_t out_cap, int64_t *n_out);
/* The same with tri- and tetra-allelic sites beside the biallelic ones (the
 * reference's gt3 / gt4): mg[s * mstride + v] is sample s's genotype index at
 * multi-allelic site v in the VCF order (j (j + 1) / 2 + i, 255 = missing),
 * malleles[v] its allele count (3 or 4), maf_in (n_multi x 4, or NULL) its
 * allele frequencies.  Every site any sample misses is dropped; M counts the
 * biallelic and multi-allelic sites used. */
int kor_cls_relatedness_ma(const uint8_t *codes, int64_t n_samples, int64_t n_sites, int64_t stride,
                           const double *af_in, const uint8_t *mg, int64_t n_multi, int64_t mstride,
                           const uint8_t *malleles, const double *maf_in, int64_t num_samples,
                           uint64_t iterations, int threads, kor_output *out, int64_t out_cap,
                           int64_t *n_out);
/* The GL/PL estimator on soft genotype likelihoods (src/wrapper.rs:89-330):
 * gl2 / gl3 / gl4 hold n2 / n3 / n4 sites of 2 / 3 / 4 alleles, each
 * n_samples x G linear-scale likelihoods (G = 3, 6, 10, genotypes in the VCF
 * order; a row with a NaN is a missing sample).  Allele frequencies come from
 * the per-site HWE SQP with the maf cut (maf < 0 or NaN: 1 / (2 n_samples)),
 * alleles of zero frequency are dropped (a site left with one allele goes), and
 * each pair's rows are sum over genotype pairs of GLx GLy m[gx][gy].  Rows as
 * kor_relatedness.  af_out (optional, 4 per site in input order) gets the
 * fitted frequencies. */
int kor_gl_relatedness(const double *gl2, int64_t n2, const double *gl3, int64_t n3, const double *gl4,
                       int64_t n4, int64_t n_samples, double maf, int64_t num_samples, uint64_t iterations,
                       int threads, kor_output *out, int64_t out_cap, int64_t *n_out, double *af_out);
/* The per-site allele-frequency fit alone (src/allele/mod.rs:91-134): gl is
 * n_sites x n_samples x G; af_out n_sites x 4. */
int kor_gl_allele_frequencies(const double *gl, int64_t n_sites, int64_t n_samples, int n_alleles,
                              uint64_t iterations, double maf, int threads, double *af_out);
/* m[gx][gy] of a site with allele frequencies freq (genotype indices in the VCF
 * order): the nine conditional probabilities of the joint genotypes. */
void kor_iis_row(int gx, int gy, const double *freq, double row[9]);
/* Pass counters of the last kor_relatedness_pairs call on this thread group:
 * total grad/Hessian passes and objective passes summed over pairs. */
void kor_pass_counts(uint64_t *gh_passes, uint64_t *obj_passes);

#ifdef __cplusplus
}
#endif

#endif
