/*
 * kestrel_oracle.c — TEST INFRASTRUCTURE ONLY (checker and CPU baseline).
 *
 * FP64 CPU restatement of malariagen/kestrel's maximum-likelihood Jacquard
 * estimator on hard calls.  Only tests, the smoke check and the benchmark's CPU
 * baseline leg load this library; the product never does.
 *
 * Parity: UNPINNED by the reference (Rust, not buildable here; no golden
 * vectors exist for this path).  See kestrel_oracle.h.
 *
 * Layout follows the reference's AVX-512 lane path so that the timed baseline
 * does the same work in the same order: per pair the 9-wide likelihood rows of
 * the jointly observed sites are materialised once (src/coefficients.rs:99-109),
 * in blocks of 8 sites (src/lanevector.rs:99-116) plus a scalar remainder, then
 * every SQP evaluation streams that buffer.  Eight f64 lanes are held as two AVX2
 * registers (x86-64-v3, the reference's published wheel baseline, README.md:20)
 * with explicit FMAs where the reference uses mul_add/fmadd and plain mul/add
 * elsewhere; compile with -ffp-contract=off so no other contraction happens.
 *
 * Deliberate differences from the reference, all below the tolerances used:
 *  - natural log is libm's log() instead of the sleef-derived log of
 *    src/log/scalar.rs:18-58 (both within about 1 ulp);
 *  - one-hot rows are exact (zeros stay zero), whereas the reference's PL=255
 *    encoding leaves ~1e-26 residues (changes f, g, H by < 1e-18 relative);
 *  - the per-site HWE SQP of the allele frequencies (src/allele/mod.rs:78-134)
 *    sums its terms per genotype class (count x term) rather than per sample.
 */
#include "kestrel_oracle.h"

#include <immintrin.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------- tuneables */
/* src/sqp.rs:31-46 with the ML path's QP iteration cap of 10
 * (src/coefficients.rs:73). */
typedef struct {
    uint64_t sqp_max_iter;
    double sqp_conv_tol;
    uint64_t qp_max_iter;
    double qp_conv_tol;
    double qp_zero_search_tol;
    uint64_t bls_max_iter;
    double bls_sufficient_decrease;
    double bls_step_size_reduce;
    double epsilon;
} tune_t;

static tune_t make_tune(uint64_t sqp_iters) {
    tune_t t;
    t.sqp_max_iter = sqp_iters;
    t.sqp_conv_tol = 1e-8;
    t.qp_max_iter = 10;
    t.qp_conv_tol = 1e-10;
    t.qp_zero_search_tol = 1e-12;
    t.bls_max_iter = 10;
    t.bls_sufficient_decrease = 1e-4;
    t.bls_step_size_reduce = 0.9;
    t.epsilon = 1e-8;
    return t;
}

/* ------------------------------------------------------- 8-lane f64 vectors */
typedef struct { __m256d lo, hi; } v8d;

static inline v8d v8_set1(double a) { v8d r; r.lo = _mm256_set1_pd(a); r.hi = r.lo; return r; }
static inline v8d v8_zero(void) { v8d r; r.lo = _mm256_setzero_pd(); r.hi = r.lo; return r; }
static inline v8d v8_add(v8d a, v8d b) { v8d r; r.lo = _mm256_add_pd(a.lo, b.lo); r.hi = _mm256_add_pd(a.hi, b.hi); return r; }
static inline v8d v8_mul(v8d a, v8d b) { v8d r; r.lo = _mm256_mul_pd(a.lo, b.lo); r.hi = _mm256_mul_pd(a.hi, b.hi); return r; }
static inline v8d v8_div(v8d a, v8d b) { v8d r; r.lo = _mm256_div_pd(a.lo, b.lo); r.hi = _mm256_div_pd(a.hi, b.hi); return r; }
/* a*b + c, fused */
static inline v8d v8_fma(v8d a, v8d b, v8d c) {
    v8d r; r.lo = _mm256_fmadd_pd(a.lo, b.lo, c.lo); r.hi = _mm256_fmadd_pd(a.hi, b.hi, c.hi); return r;
}
/* Horizontal sum in the halving order of an AVX-512 reduce. */
static inline double v8_radd(v8d a) {
    __m256d s = _mm256_add_pd(a.lo, a.hi);
    __m128d t = _mm_add_pd(_mm256_castpd256_pd128(s), _mm256_extractf128_pd(s, 1));
    return _mm_cvtsd_f64(t) + _mm_cvtsd_f64(_mm_unpackhi_pd(t, t));
}
static inline v8d v8_log(v8d a) {
    double t[8];
    _mm256_storeu_pd(t, a.lo);
    _mm256_storeu_pd(t + 4, a.hi);
    for (int i = 0; i < 8; i++) t[i] = log(t[i]);
    v8d r; r.lo = _mm256_loadu_pd(t); r.hi = _mm256_loadu_pd(t + 4); return r;
}

/* --------------------------------------------------------- likelihood rows */
/* One-hot form of the biallelic conditional genotype-pair likelihood
 * (src/mixture.rs:96-236; the same table as src/iis.rs:279-462 for two alleles).
 * gx, gy in {0,1,2}; p = REF frequency, q = ALT frequency.  The products are
 * formed in the reference's order so that the rows match bit for bit. */
static void likelihood_row(int gx, int gy, double p, double q, double row[9]) {
    double p2 = p * p, p3 = p2 * p, q2 = q * q, q3 = q2 * q;
    double pq = p * q, p2q = p2 * q, pq2 = p * q2, p2q2 = p2 * q2;
    double p3q = p3 * q, pq3 = p * q3;
    double twopq = pq + pq, twop2q = p2q + p2q, twop3q = p3q + p3q;
    double twopq2 = pq2 + pq2, twopq3 = pq3 + pq3;
    for (int k = 0; k < 9; k++) row[k] = 0.0;
    switch (gx * 3 + gy) {
    case 0: /* (0/0, 0/0) */
        row[0] = p; row[1] = p2; row[2] = p2; row[3] = p3; row[4] = p2;
        row[5] = p3; row[6] = p2; row[7] = p3; row[8] = p2 * p2; break;
    case 1: /* (0/0, 0/1) */
        row[2] = pq; row[3] = twop2q; row[7] = p2q; row[8] = twop3q; break;
    case 2: /* (0/0, 1/1) */
        row[1] = pq; row[3] = pq2; row[5] = p2q; row[8] = p2q2; break;
    case 3: /* (0/1, 0/0) */
        row[4] = pq; row[5] = twop2q; row[7] = p2q; row[8] = twop3q; break;
    case 4: /* (0/1, 0/1) */
        row[6] = twopq; row[7] = pq; row[8] = twopq * twopq; break;
    case 5: /* (0/1, 1/1) */
        row[4] = pq; row[5] = twopq2; row[7] = pq2; row[8] = twopq3; break;
    case 6: /* (1/1, 0/0) */
        row[1] = pq; row[3] = p2q; row[5] = pq2; row[8] = p2q2; break;
    case 7: /* (1/1, 0/1) */
        row[2] = pq; row[3] = twopq2; row[7] = pq2; row[8] = twopq3; break;
    case 8: /* (1/1, 1/1) */
        row[0] = q; row[1] = q2; row[2] = q2; row[3] = q3; row[4] = q2;
        row[5] = q3; row[6] = q2; row[7] = q3; row[8] = q2 * q2; break;
    }
}

/* Row buffer: full blocks of 8 sites (column-major within a block) plus up to 7
 * remainder rows, as the reference's LaneVector<_, 9>. */
typedef struct {
    v8d *blocks;      /* n_blocks * 9 */
    int64_t n_blocks;
    double rem[8][9];
    int n_rem;
    double cur[9][8];
    int cur_rows;
} rowbuf_t;

static void rb_reset(rowbuf_t *rb) { rb->n_blocks = 0; rb->n_rem = 0; rb->cur_rows = 0; }

static void rb_push(rowbuf_t *rb, const double row[9]) {
    for (int k = 0; k < 9; k++) rb->cur[k][rb->cur_rows] = row[k];
    if (++rb->cur_rows == 8) {
        v8d *b = rb->blocks + rb->n_blocks * 9;
        for (int k = 0; k < 9; k++) {
            b[k].lo = _mm256_loadu_pd(&rb->cur[k][0]);
            b[k].hi = _mm256_loadu_pd(&rb->cur[k][4]);
        }
        rb->n_blocks++;
        rb->cur_rows = 0;
    }
}

static void rb_finish(rowbuf_t *rb) {
    for (int i = 0; i < rb->cur_rows; i++)
        for (int k = 0; k < 9; k++) rb->rem[i][k] = rb->cur[k][i];
    rb->n_rem = rb->cur_rows;
    rb->cur_rows = 0;
}

static int64_t rb_len(const rowbuf_t *rb) { return rb->n_blocks * 8 + rb->n_rem; }

/* ------------------------------------------------------------ f, g and H */
/* Objective -(1/n) sum log(eps + L.x)  (src/jacquard/objective.rs:9-52). */
static double pair_objective(const rowbuf_t *rb, const double x[9], double eps) {
    v8d zx[9];
    for (int i = 0; i < 9; i++) zx[i] = v8_set1(x[i]);
    v8d zs = v8_zero(), ze = v8_set1(eps);
    for (int64_t b = 0; b < rb->n_blocks; b++) {
        const v8d *c = rb->blocks + b * 9;
        v8d d = ze;
        for (int col = 0; col < 9; col++) d = v8_fma(zx[col], c[col], d);
        zs = v8_add(zs, v8_log(d));
    }
    double sb = v8_radd(zs);
    double sr = 0.0;
    for (int i = 0; i < rb->n_rem; i++) {
        double d = eps;
        for (int col = 0; col < 9; col++) d = fma(x[col], rb->rem[i][col], d);
        sr = sr + log(d);
    }
    return -(sb + sr) / (double)rb_len(rb);
}

#define TILE_BLOCKS 32

/* Gradient and upper-triangular Hessian over 8-lane blocks, in tiles of 32
 * blocks: per tile the partial sums start at zero and are then added to the
 * running totals (src/jacquard/grad_hess.rs:44-146 and its three Hessian
 * sub-passes, which do not change any entry's summation order). */
static void gh_blocks(const v8d *blocks, int64_t n_blocks, const double x[9], double eps,
                      double g_out[9], double h_out[45]) {
    v8d g[9], h[45], zx[9], buf[TILE_BLOCKS][9];
    for (int i = 0; i < 9; i++) { g[i] = v8_zero(); zx[i] = v8_set1(x[i]); }
    for (int i = 0; i < 45; i++) h[i] = v8_zero();
    v8d one = v8_set1(1.0), ze = v8_set1(eps);
    for (int64_t t0 = 0; t0 < n_blocks; t0 += TILE_BLOCKS) {
        int nb = (int)((n_blocks - t0) < TILE_BLOCKS ? (n_blocks - t0) : TILE_BLOCKS);
        v8d zg[9];
        for (int k = 0; k < 9; k++) zg[k] = v8_zero();
        for (int i = 0; i < nb; i++) {
            const v8d *c = blocks + (t0 + i) * 9;
            v8d d = ze;
            for (int col = 0; col < 9; col++) d = v8_fma(zx[col], c[col], d);
            d = v8_div(one, d);
            for (int col = 0; col < 9; col++) zg[col] = v8_fma(c[col], d, zg[col]);
            for (int col = 0; col < 9; col++) buf[i][col] = v8_mul(c[col], d);
        }
        for (int k = 0; k < 9; k++) g[k] = v8_add(g[k], zg[k]);
        int id = 0;
        for (int a = 0; a < 9; a++) {
            for (int b = a; b < 9; b++, id++) {
                v8d z = v8_zero();
                for (int i = 0; i < nb; i++) z = v8_fma(buf[i][a], buf[i][b], z);
                h[id] = v8_add(h[id], z);
            }
        }
    }
    for (int k = 0; k < 9; k++) g_out[k] = v8_radd(g[k]);
    for (int k = 0; k < 45; k++) h_out[k] = v8_radd(h[k]);
}

/* The scalar (one-lane) form of the same loop, used for the remainder rows. */
static void gh_rem(const double (*rows)[9], int n_rows, const double x[9], double eps,
                   double g_out[9], double h_out[45]) {
    double g[9] = {0}, h[45] = {0};
    double buf[TILE_BLOCKS][9];
    for (int t0 = 0; t0 < n_rows; t0 += TILE_BLOCKS) {
        int nb = (n_rows - t0) < TILE_BLOCKS ? (n_rows - t0) : TILE_BLOCKS;
        double zg[9] = {0};
        for (int i = 0; i < nb; i++) {
            const double *c = rows[t0 + i];
            double d = eps;
            for (int col = 0; col < 9; col++) d = fma(x[col], c[col], d);
            d = 1.0 / d;
            for (int col = 0; col < 9; col++) zg[col] = fma(c[col], d, zg[col]);
            for (int col = 0; col < 9; col++) buf[i][col] = c[col] * d;
        }
        for (int k = 0; k < 9; k++) g[k] = g[k] + zg[k];
        int id = 0;
        for (int a = 0; a < 9; a++) {
            for (int b = a; b < 9; b++, id++) {
                double z = 0.0;
                for (int i = 0; i < nb; i++) z = fma(buf[i][a], buf[i][b], z);
                h[id] = h[id] + z;
            }
        }
    }
    memcpy(g_out, g, sizeof g);
    memcpy(h_out, h, sizeof h);
}

/* src/jacquard/grad_hess.rs:13-41: g = -(sum L d)/n, H = (sum (Ld)(Ld)^T)/n. */
static void pair_grad_hess(const rowbuf_t *rb, const double x[9], double eps,
                           double g[9], double H[9][9]) {
    double bg[9], bh[45], rg[9], rh[45];
    gh_blocks(rb->blocks, rb->n_blocks, x, eps, bg, bh);
    gh_rem((const double (*)[9])rb->rem, rb->n_rem, x, eps, rg, rh);
    double n = (double)rb_len(rb);
    for (int i = 0; i < 9; i++) g[i] = -(bg[i] + rg[i]) / n;
    int id = 0;
    for (int i = 0; i < 9; i++)
        for (int j = i; j < 9; j++, id++) {
            double v = (bh[id] + rh[id]) / n;
            H[i][j] = v;
            H[j][i] = v;
        }
}

/* ------------------------------------------------------ small dense algebra */
/* src/algebra.rs:4-84 */
static double dotn(int n, const double *a, const double *b) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s = fma(a[i], b[i], s);
    return s;
}
static double sumn(int n, const double *a) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i];
    return s;
}
static void sum_to_one_n(int n, const double *x, double *out) {
    double s = sumn(n, x);
    for (int i = 0; i < n; i++) out[i] = x[i] / s;
}
static void sum_to_one(const double *x, double *out) { sum_to_one_n(9, x, out); }
static void matvec(int n, const double M[9][9], const double *v, double *out) {
    for (int i = 0; i < n; i++) out[i] = dotn(n, M[i], v);
}

/* ---------------------------------------------------------- LDL^T helpers */
/* src/cholesky.rs:6-65, GMW81 modified LDL^T. */
static void ldl_modified(int n, const double a[9][9], double l[9][9], double d[9]) {
    double gamma = 0.0, xi = 0.0;
    for (int i = 0; i < n; i++) gamma = fmax(gamma, fabs(a[i][i]));
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) xi = fmax(xi, fabs(a[i][j]));
    const double eps = 2.220446049250313e-16;
    double delta = eps * fmax(1.0, gamma + xi);
    double t = sqrt((double)n * (double)n - 1.0);
    double ratio = n <= 1 ? 0.0 : xi / t;
    double beta2 = fmax(fmax(gamma, ratio), eps);
    double pv[9];
    for (int j = 0; j < n; j++) {
        double sjj = 0.0;
        for (int s = 0; s < j; s++) {
            pv[s] = d[s] * l[j][s];
            sjj = fma(pv[s], l[j][s], sjj);
        }
        double cjj = a[j][j] - sjj;
        l[j][j] = 1.0;
        double theta = 0.0;
        for (int i = j + 1; i < n; i++) {
            double sij = 0.0;
            for (int s = 0; s < j; s++) sij = fma(pv[s], l[i][s], sij);
            double cij = a[i][j] - sij;
            theta = fmax(theta, fabs(cij));
            l[i][j] = cij;
        }
        double dj = fmax(fmax(fabs(cjj), theta * theta / beta2), delta);
        for (int i = j + 1; i < n; i++) l[i][j] /= dj;
        d[j] = dj;
    }
}

/* src/cholesky.rs:72-102, plain LDL^T. */
static void ldl_plain(int n, const double a[9][9], double l[9][9], double d[9]) {
    double pv[9];
    for (int j = 0; j < n; j++) {
        l[j][j] = 1.0;
        double sjj = 0.0;
        for (int s = 0; s < j; s++) {
            pv[s] = d[s] * l[j][s];
            sjj = fma(pv[s], l[j][s], sjj);
        }
        double dj = a[j][j] - sjj;
        for (int i = j + 1; i < n; i++) {
            double sij = 0.0;
            for (int s = 0; s < j; s++) sij = fma(pv[s], l[i][s], sij);
            l[i][j] = (a[i][j] - sij) / dj;
        }
        d[j] = dj;
    }
}

static void fwd_unit(int n, const double l[9][9], double *b) {
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = 0; j < i; j++) s = fma(b[j], l[i][j], s);
        b[i] -= s;
    }
}
static void bwd_unit(int n, const double l[9][9], double *b) {
    for (int i = n - 1; i >= 0; i--) {
        double s = 0.0;
        for (int j = i + 1; j < n; j++) s = fma(b[j], l[j][i], s);
        b[i] -= s;
    }
}
static void ldl_solve(int n, const double l[9][9], const double *d, double *b) {
    fwd_unit(n, l, b);
    for (int i = 0; i < n; i++) b[i] /= d[i];
    bwd_unit(n, l, b);
}

/* ------------------------------------------------------------------- SQP */
/* src/sqp.rs:95-109 */
static int kkt_converged(const double x[9], const double g[9], double tol) {
    double lambda = dotn(9, x, g);
    for (int i = 0; i < 9; i++) {
        if (x[i] == 0.0) {
            if (!(g[i] >= lambda - tol)) return 0;
        } else {
            if (!(fabs(g[i] - lambda) <= tol)) return 0;
        }
    }
    return 1;
}

/* src/sqp.rs:252-268 */
static double feasible_step_n(int n, const double y[9], const double p[9], int *block) {
    double alpha = 1.0;
    *block = -1;
    for (int i = 0; i < n; i++) {
        if (p[i] < 0.0) {
            double a = -y[i] / p[i];
            if (a < alpha) { alpha = a; *block = i; }
        }
    }
    return alpha;
}

/* Active-set QP on the simplex of dimension n <= 9, src/sqp.rs:112-250
 * (modify = true; the reference's const generic N is n here).  Returns the
 * iteration count the reference returns beside y. */
static uint64_t qp_active_set_n(int n, const double Q[9][9], const double c[9], const double y0[9],
                                const tune_t *tu, double y_out[9]) {
    double y[9] = {0};
    int work[9] = {0};
    memcpy(y, y0, sizeof(double) * n);
    for (int i = 0; i < n; i++) work[i] = (y[i] == 0.0);
    uint64_t it = 0;
    while (it < tu->qp_max_iter) {
        double ys[9];
        sum_to_one_n(n, y, ys);
        memcpy(y, ys, sizeof(double) * n);
        int fi[9], nf = 0;
        for (int i = 0; i < n; i++) if (!work[i]) fi[nf++] = i;
        if (nf == 0) abort(); /* the reference asserts here */
        double yf[9] = {0}, cf[9] = {0}, Qf[9][9] = {{0}};
        for (int i = 0; i < nf; i++) {
            yf[i] = y[fi[i]];
            cf[i] = c[fi[i]];
            for (int j = 0; j < nf; j++) Qf[i][j] = Q[fi[i]][fi[j]];
        }
        double qy[9], gf[9] = {0};
        matvec(nf, Qf, yf, qy);
        for (int i = 0; i < nf; i++) gf[i] = cf[i] + qy[i];
        double L[9][9] = {{0}}, D[9] = {0};
        ldl_modified(nf, Qf, L, D);
        ldl_solve(nf, L, D, gf);
        double ones[9] = {0};
        for (int i = 0; i < nf; i++) ones[i] = 1.0;
        ldl_solve(nf, L, D, ones);
        double lambda = sumn(nf, gf) / sumn(nf, ones);
        /* The reference forms lambda*ones - g over all N slots; the slots past
         * nf are zero on both sides. */
        double m = 0.0;
        for (int i = 0; i < n; i++) {
            gf[i] = lambda * ones[i] - gf[i];
            double a = fabs(gf[i]);
            /* a total order that ranks NaN above everything, as total_cmp does */
            if (isnan(a) || isnan(m)) m = NAN;
            else if (a > m) m = a;
        }
        if (m <= tu->qp_zero_search_tol) {
            if (nf == n) { memcpy(y_out, y, sizeof(double) * n); return it; }
            double qy9[9], gq[9];
            matvec(n, Q, y, qy9);
            for (int i = 0; i < n; i++) gq[i] = c[i] + qy9[i];
            int best = -1;
            for (int i = 0; i < n; i++)
                if (work[i] && (best < 0 || gq[i] < gq[best])) best = i;
            double mult = gq[best] - lambda;
            if (mult >= -tu->qp_conv_tol) { memcpy(y_out, y, sizeof(double) * n); return it; }
            work[best] = 0;
        } else {
            double p[9] = {0};
            int k = 0;
            for (int i = 0; i < n; i++) if (!work[i]) p[i] = gf[k++];
            int block;
            double alpha = feasible_step_n(n, y, p, &block);
            for (int i = 0; i < n; i++) y[i] = fmax(y[i] + alpha * p[i], 0.0);
            if (block >= 0) { work[block] = 1; y[block] = 0.0; }
        }
        it++;
    }
    memcpy(y_out, y, sizeof(double) * n);
    return it;
}

static void qp_active_set(const double Q[9][9], const double c[9], const double y0[9],
                          const tune_t *tu, double y_out[9]) {
    (void)qp_active_set_n(9, Q, c, y0, tu, y_out);
}

/* Reduced-Hessian condition estimate, src/sqp.rs:313-391. */
static double condition_estimate(const double x[9], const double g[9], const double H[9][9], double tol) {
    double lambda = dotn(9, x, g);
    int fi[9], nf = 0;
    for (int i = 0; i < 9; i++) {
        int strict = (x[i] == 0.0) && (g[i] >= lambda + tol);
        if (!strict) fi[nf++] = i;
    }
    if (nf == 0) abort();
    double Hf[9][9] = {{0}};
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) Hf[i][j] = H[fi[i]][fi[j]];
    double L[9][9] = {{0}}, D[9] = {0};
    ldl_plain(nf, Hf, L, D);
    for (int i = 0; i < nf; i++) if (!(D[i] > 0.0)) return INFINITY;
    /* First maximum / first minimum by value (a total order on positives). */
    int imax = 0, imin = 0;
    for (int i = 1; i < nf; i++) {
        if (D[i] >= D[imax]) imax = i;   /* max_by keeps the last of equals */
        if (D[i] < D[imin]) imin = i;    /* min_by keeps the first of equals */
    }
    double emax[9] = {0}, emin[9] = {0};
    emax[imax] = 1.0;
    emin[imin] = 1.0;
    double wmax[9] = {0};
    matvec(nf, L, emax, wmax);
    bwd_unit(nf, L, emin);
    double nmax = sqrt(dotn(nf, wmax, wmax));
    double nmin = sqrt(dotn(nf, emin, emin));
    return nmax * nmin * (D[imax] / D[imin]);
}

typedef struct {
    uint64_t gh;
    uint64_t obj;
} pass_count_t;

/* src/sqp.rs:270-310 */
static double line_search(const rowbuf_t *rb, const double x[9], const double y[9],
                          const double g[9], double f, const tune_t *tu,
                          double xnew_out[9], pass_count_t *pc) {
    double p[9];
    for (int i = 0; i < 9; i++) p[i] = y[i] - x[i];
    double t = tu->bls_sufficient_decrease * dotn(9, g, p);
    double alpha = 1.0;
    uint64_t it = 0;
    for (;;) {
        double xn[9], xs[9];
        for (int i = 0; i < 9; i++) xn[i] = x[i] + alpha * p[i];
        sum_to_one(xn, xs);
        double fn = pair_objective(rb, xs, tu->epsilon);
        pc->obj++;
        if (fn <= f + alpha * t) { memcpy(xnew_out, xs, sizeof xs); return fn; }
        it++;
        if (it == tu->bls_max_iter) { memcpy(xnew_out, xs, sizeof xs); return fn; }
        alpha *= tu->bls_step_size_reduce;
    }
}

/* src/sqp.rs:49-93 */
static void solve_sqp(const rowbuf_t *rb, const double x0[9], const tune_t *tu,
                      kor_output *o, pass_count_t *pc) {
    double x[9];
    sum_to_one(x0, x);
    double f = pair_objective(rb, x, tu->epsilon);
    pc->obj++;
    for (uint64_t it = 0; it < tu->sqp_max_iter; it++) {
        double g[9], H[9][9];
        pair_grad_hess(rb, x, tu->epsilon, g, H);
        pc->gh++;
        if (kkt_converged(x, g, tu->sqp_conv_tol)) {
            o->cond = condition_estimate(x, g, H, tu->sqp_conv_tol);
            memcpy(o->jacquard, x, sizeof x);
            o->obj = f;
            o->iters = it;
            return;
        }
        double hx[9], c[9], y[9], xn[9];
        matvec(9, H, x, hx);
        for (int i = 0; i < 9; i++) c[i] = g[i] - hx[i];
        qp_active_set(H, c, x, tu, y);
        f = line_search(rb, x, y, g, f, tu, xn, pc);
        memcpy(x, xn, sizeof x);
    }
    memcpy(o->jacquard, x, sizeof x);
    o->obj = f;
    o->iters = tu->sqp_max_iter;
    o->cond = NAN;
}

/* ---------------------------------------------------------- frequencies */
int kor_allele_counts(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                      int64_t stride, int32_t *ref_count, int32_t *obs_count) {
    if (!codes || n_samples <= 0 || n_sites <= 0 || stride < n_sites) return KOR_EINVAL;
    for (int64_t s = 0; s < n_sites; s++) { ref_count[s] = 0; obs_count[s] = 0; }
    for (int64_t i = 0; i < n_samples; i++) {
        const uint8_t *r = codes + i * stride;
        for (int64_t s = 0; s < n_sites; s++) {
            uint8_t c = r[s];
            if (c > 3) return KOR_EINVAL;
            if (c != 3) { ref_count[s] += 2 - c; obs_count[s] += 1; }
        }
    }
    return KOR_OK;
}

/* A biallelic site's frequencies from its hard calls: the reference's GL path
 * on one-hot likelihoods, i.e. the per-site HWE SQP of src/allele/mod.rs:91-134
 * (defined with the soft-likelihood code below) on the three genotype classes
 * weighted by their counts, then the maf cut. */
static void hard_call_frequencies(const int64_t cnt[3], uint64_t iterations, double maf, double f[4]);

int kor_site_frequencies(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                         int64_t stride, const double *af_in, double maf,
                         double *p, double *q, uint8_t *keep, int64_t *n_kept) {
    return kor_site_frequencies_it(codes, n_samples, n_sites, stride, af_in, maf, 100, p, q, keep, n_kept);
}

int kor_site_frequencies_it(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                            int64_t stride, const double *af_in, double maf, uint64_t iterations,
                            double *p, double *q, uint8_t *keep, int64_t *n_kept) {
    if (n_samples <= 0 || n_sites <= 0 || iterations == 0) return KOR_EINVAL;
    int64_t kept = 0;
    if (af_in) {
        for (int64_t s = 0; s < n_sites; s++) {
            p[s] = af_in[2 * s];
            q[s] = af_in[2 * s + 1];
            keep[s] = (p[s] > 0.0 && q[s] > 0.0);
            kept += keep[s];
        }
        *n_kept = kept;
        return KOR_OK;
    }
    if (maf < 0.0) maf = 1.0 / (2.0 * (double)n_samples);
    for (int64_t s = 0; s < n_sites; s++) {
        int64_t cnt[3] = {0, 0, 0};
        for (int64_t i = 0; i < n_samples; i++) {
            const uint8_t c = codes[i * stride + s];
            if (c > 3) return KOR_EINVAL;
            if (c < 3) cnt[c]++;
        }
        p[s] = 0.0; q[s] = 0.0; keep[s] = 0;
        if (cnt[0] + cnt[1] + cnt[2] == 0) continue; /* no observed call: nothing to estimate */
        double f[4];
        hard_call_frequencies(cnt, iterations, maf, f);
        p[s] = f[0];
        q[s] = f[1];
        keep[s] = (f[0] > 0.0 && f[1] > 0.0);
        kept += keep[s];
    }
    *n_kept = kept;
    return KOR_OK;
}

/* ------------------------------------------------------------- drivers */
static void build_rows(rowbuf_t *rb, const uint8_t *cx, const uint8_t *cy, int64_t n_sites,
                       const double *p, const double *q, const uint8_t *keep) {
    rb_reset(rb);
    double row[9];
    for (int64_t s = 0; s < n_sites; s++) {
        if (!keep[s]) continue;
        int gx = cx[s], gy = cy[s];
        if (gx == 3 || gy == 3) continue;
        likelihood_row(gx, gy, p[s], q[s], row);
        rb_push(rb, row);
    }
    rb_finish(rb);
}

static uint64_t g_last_gh, g_last_obj;

void kor_pass_counts(uint64_t *gh, uint64_t *obj) {
    *gh = g_last_gh;
    *obj = g_last_obj;
}

int kor_relatedness_pairs(const uint8_t *codes, int64_t n_sites, int64_t stride,
                          const double *p, const double *q, const uint8_t *keep,
                          const int64_t *pair_x, const int64_t *pair_y,
                          int64_t n_pairs, uint64_t iterations, int threads,
                          kor_output *out) {
    if (!codes || !p || !q || !keep || n_sites <= 0 || iterations == 0) return KOR_EINVAL;
    tune_t tu = make_tune(iterations);
    int err = KOR_OK;
    uint64_t tot_gh = 0, tot_obj = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads) reduction(+ : tot_gh, tot_obj)
#endif
    {
        rowbuf_t rb;
        rb.blocks = (v8d *)aligned_alloc(64, sizeof(v8d) * 9 * (size_t)(n_sites / 8 + 1));
        pass_count_t pc = {0, 0};
        if (!rb.blocks) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
            err = KOR_ENOMEM;
        } else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t k = 0; k < n_pairs; k++) {
                int64_t x = pair_x[k], y = pair_y[k];
                kor_output *o = out + k;
                o->x = (uint64_t)x;
                o->y = (uint64_t)y;
                build_rows(&rb, codes + x * stride, codes + y * stride, n_sites, p, q, keep);
                if (rb_len(&rb) == 0) {
#ifdef _OPENMP
#pragma omp atomic write
#endif
                    err = KOR_ENOSITES;
                    memset(o->jacquard, 0, sizeof o->jacquard);
                    o->obj = NAN; o->iters = 0; o->cond = NAN;
                    continue;
                }
                double x0[9];
                if (x == y) {
                    for (int i = 0; i < 9; i++) x0[i] = 0.0;
                    x0[0] = 0.5;
                    x0[6] = 0.5;
                } else {
                    for (int i = 0; i < 9; i++) x0[i] = 1.0 / 9.0;
                }
                solve_sqp(&rb, x0, &tu, o, &pc);
            }
            free(rb.blocks);
        }
        tot_gh += pc.gh;
        tot_obj += pc.obj;
    }
    g_last_gh = tot_gh;
    g_last_obj = tot_obj;
    return err;
}

int kor_relatedness(const uint8_t *codes, int64_t n_samples, int64_t n_sites,
                    int64_t stride, const double *af_in, int64_t num_samples,
                    uint64_t iterations, double maf, int threads,
                    kor_output *out, int64_t out_cap, int64_t *n_out) {
    if (!codes || n_samples <= 0 || n_sites <= 0 || stride < n_sites) return KOR_EINVAL;
    if (num_samples < 0) num_samples = n_samples;
    if (num_samples > n_samples) return KOR_EINVAL;
    int64_t npairs = num_samples * (num_samples + 1) / 2;
    if (out_cap < npairs) return KOR_EINVAL;
    double *p = (double *)malloc(sizeof(double) * n_sites);
    double *q = (double *)malloc(sizeof(double) * n_sites);
    uint8_t *keep = (uint8_t *)malloc(n_sites);
    int64_t *px = (int64_t *)malloc(sizeof(int64_t) * (npairs ? npairs : 1));
    int64_t *py = (int64_t *)malloc(sizeof(int64_t) * (npairs ? npairs : 1));
    int st = KOR_ENOMEM;
    if (p && q && keep && px && py) {
        int64_t kept;
        st = kor_site_frequencies_it(codes, n_samples, n_sites, stride, af_in, maf, iterations, p, q, keep, &kept);
        if (st == KOR_OK && kept == 0) st = KOR_ENOSITES;
        if (st == KOR_OK) {
            int64_t k = 0;
            for (int64_t x = 0; x < num_samples; x++)
                for (int64_t y = x; y < num_samples; y++) { px[k] = x; py[k] = y; k++; }
            st = kor_relatedness_pairs(codes, n_sites, stride, p, q, keep, px, py, npairs,
                                       iterations, threads, out);
            *n_out = npairs;
        }
    }
    free(p); free(q); free(keep); free(px); free(py);
    return st;
}

int kor_eval_pair(const uint8_t *codes_x, const uint8_t *codes_y, int64_t n_sites,
                  const double *p, const double *q, const uint8_t *keep,
                  const double delta[9], double *f, double g[9], double h[81],
                  int64_t *n_used) {
    rowbuf_t rb;
    rb.blocks = (v8d *)aligned_alloc(64, sizeof(v8d) * 9 * (size_t)(n_sites / 8 + 1));
    if (!rb.blocks) return KOR_ENOMEM;
    build_rows(&rb, codes_x, codes_y, n_sites, p, q, keep);
    *n_used = rb_len(&rb);
    if (*n_used == 0) { free(rb.blocks); return KOR_ENOSITES; }
    *f = pair_objective(&rb, delta, 1e-8);
    double H[9][9];
    pair_grad_hess(&rb, delta, 1e-8, g, H);
    memcpy(h, H, sizeof H);
    free(rb.blocks);
    return KOR_OK;
}

/* ------------------------------------------- GT conditional least squares */
/* m[gx][gy] of one biallelic site, src/iis.rs:279-462 with the biallelic IIS
 * modes of src/conditional.rs:6-55 (allele 0 = REF with frequency p, 1 = ALT
 * with q), products in the reference's order. */
static void cls_row(int gx, int gy, double p, double q, double row[9]) {
    for (int k = 0; k < 9; k++) row[k] = 0.0;
    switch (gx * 3 + gy) {
    case 0: case 8: { /* M1 ii-ii, pi = p or q */
        const double pi = gx == 0 ? p : q, pi2 = pi * pi, pi3 = pi2 * pi;
        row[0] = pi; row[1] = pi2; row[2] = pi2; row[3] = pi3; row[4] = pi2;
        row[5] = pi3; row[6] = pi2; row[7] = pi3; row[8] = pi2 * pi2; break;
    }
    case 2: case 6: { /* M2 ii-kk */
        const double pi = gx == 0 ? p : q, pk = gx == 0 ? q : p;
        const double pi2 = pi * pi, pk2 = pk * pk;
        row[1] = pi * pk; row[3] = pi * pk2; row[5] = pi2 * pk; row[8] = pi2 * pk2; break;
    }
    case 1: case 7: { /* M3 ii-il (0/0, 0/1: pl = q) and M4 ii-ki (1/1, 0/1: pk = p) */
        const double pi = gx == 0 ? p : q, po = gx == 0 ? q : p;
        const double pi2 = pi * pi, pi3 = pi2 * pi;
        row[2] = pi * po; row[3] = (2.0 * pi2) * po; row[7] = pi2 * po; row[8] = (2.0 * pi3) * po; break;
    }
    case 3: { /* M6 ij-ii: pi = p, pj = q */
        const double pi = p, pj = q, pi2 = pi * pi, pi3 = pi2 * pi;
        row[4] = pi * pj; row[5] = (2.0 * pi2) * pj; row[7] = pi2 * pj; row[8] = (2.0 * pi3) * pj; break;
    }
    case 5: { /* M7 ij-jj: pi = p, pj = q */
        const double pi = p, pj = q, pj2 = pj * pj;
        row[4] = pi * pj; row[5] = (2.0 * pj2) * pi; row[7] = pj2 * pi; row[8] = (2.0 * (pj2 * pj)) * pi; break;
    }
    case 4: { /* M9 ij-ij */
        const double pi = p, pj = q, pi2 = pi * pi, pj2 = pj * pj;
        row[6] = (2.0 * pi) * pj; row[7] = (pi * pj) * (pi + pj); row[8] = (4.0 * pi2) * pj2; break;
    }
    }
}

/* The two alleles (i <= j) of genotype index g in the VCF order
 * (j (j + 1) / 2 + i, src/coefficients.rs:19-38). */
static void genotype_alleles(int g, int *i, int *j) {
    int b = 0;
    while ((b + 1) * (b + 2) / 2 <= g) b++;
    *j = b;
    *i = g - b * (b + 1) / 2;
}

/* m[gx][gy] for any number of alleles: the nine conditional probabilities
 * P(genotypes (i, j), (k, l) | Jacquard state), the table of src/iis.rs:
 * 279-462 indexed by the IIS mode of src/conditional.rs:10-50, computed here by
 * its definition.  For each ordering of each unordered genotype (one for a
 * homozygote, two for a heterozygote), alleles x1 = a1, x2 = a2, y1 = b1,
 * y2 = b2 add, per state, the product over the state's identity classes of the
 * class's allele frequency when every member carries the same allele (zero
 * otherwise).  The classes: 1 {x1 x2 y1 y2}; 2 {x1 x2}{y1 y2}; 3 {x1 x2 y1}{y2};
 * 4 {x1 x2}{y1}{y2}; 5 {x1 y1 y2}{x2}; 6 {y1 y2}{x1}{x2}; 7 {x1 y1}{x2 y2};
 * 8 {x1 y1}{x2}{y2}; 9 all apart. */
static void iis_row(int i, int j, int k, int l, const double *f, double row[9]) {
    for (int s = 0; s < 9; s++) row[s] = 0.0;
    const int nx = i == j ? 1 : 2, ny = k == l ? 1 : 2;
    for (int u = 0; u < nx; u++) {
        const int a1 = u ? j : i, a2 = u ? i : j;
        for (int w = 0; w < ny; w++) {
            const int b1 = w ? l : k, b2 = w ? k : l;
            const double fa1 = f[a1], fa2 = f[a2], fb1 = f[b1], fb2 = f[b2];
            const int xx = a1 == a2, yy = b1 == b2, s1 = a1 == b1, s2 = a2 == b2;
            if (xx && yy && s1) row[0] += fa1;
            if (xx && yy) row[1] += fa1 * fb1;
            if (xx && s1) row[2] += fa1 * fb2;
            if (xx) row[3] += fa1 * fb1 * fb2;
            if (yy && s1) row[4] += fb1 * fa2;
            if (yy) row[5] += fb1 * fa1 * fa2;
            if (s1 && s2) row[6] += fa1 * fa2;
            if (s1) row[7] += fa1 * fa2 * fb2;
            row[8] += fa1 * fa2 * fb1 * fb2;
        }
    }
}

void kor_iis_row(int gx, int gy, const double *freq, double row[9]) {
    int i, j, k, l;
    genotype_alleles(gx, &i, &j);
    genotype_alleles(gy, &k, &l);
    iis_row(i, j, k, l, freq, row);
}

/* The reference's default hard-call estimator (src/coefficients.rs:166-278 with
 * src/cls.rs:6-49 and the Gram matrix of src/quadratic.rs), for biallelic
 * sites:
 *  - a site is used only if every sample has a call (src/vcf.rs:217-221 drops
 *    the whole record otherwise); monomorphic sites stay, and there is no maf
 *    filter (src/wrapper.rs:22-40);
 *  - allele frequencies are counts / (2 n_samples) over all samples
 *    (src/wrapper.rs:412-428) unless af_in gives them;
 *  - the per-site rows m[gx][gy] are src/iis.rs:279-462 through
 *    src/cls.rs:6-25 (cls_row);
 *  - Q = (1/M) sum over sites and all nine (gx, gy) of m m^T (src/quadratic.rs:13-37);
 *  - per pair c = (sum over sites of m[gx][gy]) / (-M) (src/cls.rs:27-49,
 *    scale_div of src/algebra.rs:61-63);
 *  - the simplex QP from 1/9 (x != y), or the two-variable QP on (Delta1,
 *    Delta7) from (1/2, 1/2) for x == y, with qp_max_iter = iterations
 *    (src/coefficients.rs:207, :231-244);
 *  - obj = delta.Q delta + 2 c.delta + 1 (Brier), iters = the QP's iteration
 *    count, cond = the reduced-Hessian estimate at g = Q delta + c
 *    (src/coefficients.rs:253-268). */
int kor_cls_relatedness(const uint8_t *codes, int64_t n_samples, int64_t n_sites, int64_t stride,
                        const double *af_in, int64_t num_samples, uint64_t iterations, int threads,
                        kor_output *out, int64_t out_cap, int64_t *n_out) {
    return kor_cls_relatedness_ma(codes, n_samples, n_sites, stride, af_in, NULL, 0, 0, NULL, NULL,
                                  num_samples, iterations, threads, out, out_cap, n_out);
}

int kor_cls_relatedness_ma(const uint8_t *codes, int64_t n_samples, int64_t n_sites, int64_t stride,
                           const double *af_in, const uint8_t *mg, int64_t n_multi, int64_t mstride,
                           const uint8_t *malleles, const double *maf_in, int64_t num_samples,
                           uint64_t iterations, int threads, kor_output *out, int64_t out_cap,
                           int64_t *n_out) {
    if (!codes || n_samples <= 0 || n_sites <= 0 || stride < n_sites || !out || !n_out || iterations == 0)
        return KOR_EINVAL;
    if (n_multi < 0 || (n_multi > 0 && (!mg || !malleles || mstride < n_multi))) return KOR_EINVAL;
    if (num_samples < 0) num_samples = n_samples;
    if (num_samples == 0 || num_samples > n_samples) return KOR_EINVAL;
    int64_t npairs = num_samples * (num_samples + 1) / 2;
    if (out_cap < npairs) return KOR_EINVAL;
    int64_t *site = (int64_t *)malloc(sizeof(int64_t) * (size_t)n_sites);
    double *p = (double *)malloc(sizeof(double) * (size_t)n_sites);
    double *q = (double *)malloc(sizeof(double) * (size_t)n_sites);
    if (!site || !p || !q) { free(site); free(p); free(q); return KOR_ENOMEM; }
    int64_t m = 0;
    for (int64_t v = 0; v < n_sites; v++) {
        int64_t refc = 0, altc = 0;
        int complete = 1;
        for (int64_t s = 0; s < n_samples; s++) {
            const uint8_t g = codes[s * stride + v];
            if (g > 2) { complete = 0; break; }
            refc += 2 - g;
            altc += g;
        }
        if (!complete) continue;
        site[m] = v;
        if (af_in) {
            p[m] = af_in[2 * v];
            q[m] = af_in[2 * v + 1];
        } else {
            const double tot = (double)(2 * n_samples);
            p[m] = (double)refc / tot;
            q[m] = (double)altc / tot;
        }
        m++;
    }
    /* tri- and tetra-allelic sites (genotype indices, 255 = missing): those
     * every sample calls; frequencies are allele counts / (2 n_samples)
     * (src/wrapper.rs:412-428) unless maf_in (n_multi x 4) gives them */
    int64_t *msite = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_multi + 1));
    double *mf = (double *)malloc(sizeof(double) * 4 * (size_t)(n_multi + 1));
    if (!msite || !mf) { free(site); free(p); free(q); free(msite); free(mf); return KOR_ENOMEM; }
    int64_t mm = 0;
    for (int64_t v = 0; v < n_multi; v++) {
        const int na = malleles[v];
        if (na < 3 || na > 4) { free(site); free(p); free(q); free(msite); free(mf); return KOR_EINVAL; }
        const int ng = na * (na + 1) / 2;
        int64_t cnt[4] = {0, 0, 0, 0};
        int complete = 1;
        for (int64_t s2 = 0; s2 < n_samples; s2++) {
            const int g = mg[s2 * mstride + v];
            if (g == 255) { complete = 0; break; }
            if (g >= ng) { free(site); free(p); free(q); free(msite); free(mf); return KOR_EINVAL; }
            int a, b;
            genotype_alleles(g, &a, &b);
            cnt[a]++;
            cnt[b]++;
        }
        if (!complete) continue;
        msite[mm] = v;
        for (int a = 0; a < 4; a++)
            mf[4 * mm + a] = maf_in ? maf_in[4 * v + a] : (a < na ? (double)cnt[a] / (double)(2 * n_samples) : 0.0);
        mm++;
    }
    if (m + mm == 0) { free(site); free(p); free(q); free(msite); free(mf); return KOR_ENOSITES; }
    const double m_total = (double)(m + mm);
    /* the Gram matrix over all sites' rows (biallelic, then the others), upper
     * triangle in the reference's row-major order (src/coefficients.rs:281-320) */
    double h[45] = {0};
    for (int64_t k = 0; k < m; k++) {
        for (int gx = 0; gx < 3; gx++)
            for (int gy = 0; gy < 3; gy++) {
                double row[9];
                cls_row(gx, gy, p[k], q[k], row);
                int a = 0;
                for (int i = 0; i < 9; i++)
                    for (int j = i; j < 9; j++) h[a++] += row[i] * row[j];
            }
    }
    for (int64_t k = 0; k < mm; k++) {
        const int na = malleles[msite[k]], ng = na * (na + 1) / 2;
        for (int gx = 0; gx < ng; gx++)
            for (int gy = 0; gy < ng; gy++) {
                double row[9];
                kor_iis_row(gx, gy, mf + 4 * k, row);
                int a = 0;
                for (int i = 0; i < 9; i++)
                    for (int j = i; j < 9; j++) h[a++] += row[i] * row[j];
            }
    }
    double Q[9][9];
    {
        int a = 0;
        for (int i = 0; i < 9; i++)
            for (int j = i; j < 9; j++) {
                const double v = h[a++] / m_total;
                Q[i][j] = v;
                Q[j][i] = v;
            }
    }
    tune_t tu = make_tune(iterations);
    tu.qp_max_iter = iterations;
    double Q2[9][9] = {{0}};
    Q2[0][0] = Q[0][0]; Q2[0][1] = Q[0][6];
    Q2[1][0] = Q[6][0]; Q2[1][1] = Q[6][6];
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
    for (int64_t x = 0; x < num_samples; x++) {
        int64_t row0 = x * num_samples - x * (x - 1) / 2;
        for (int64_t y = x; y < num_samples; y++) {
            double c[9] = {0};
            for (int64_t k = 0; k < m; k++) {
                double row[9];
                const int64_t v = site[k];
                cls_row(codes[x * stride + v], codes[y * stride + v], p[k], q[k], row);
                for (int i = 0; i < 9; i++) c[i] = c[i] + row[i];
            }
            /* c2 + (c3 + c4), src/coefficients.rs:220-224 */
            double c3[9] = {0}, c4[9] = {0};
            for (int64_t k = 0; k < mm; k++) {
                const int64_t v = msite[k];
                double row[9];
                kor_iis_row(mg[x * mstride + v], mg[y * mstride + v], mf + 4 * k, row);
                double *acc = malleles[v] == 3 ? c3 : c4;
                for (int i = 0; i < 9; i++) acc[i] = acc[i] + row[i];
            }
            for (int i = 0; i < 9; i++) c[i] = (c[i] + (c3[i] + c4[i])) / -m_total;
            double delta[9] = {0};
            uint64_t its;
            if (x == y) {
                const double x0[9] = {0.5, 0.5};
                const double c2[9] = {c[0], c[6]};
                double d2[9] = {0};
                its = qp_active_set_n(2, Q2, c2, x0, &tu, d2);
                delta[0] = d2[0];
                delta[6] = d2[1];
            } else {
                double x0[9];
                for (int i = 0; i < 9; i++) x0[i] = 1.0 / 9.0;
                its = qp_active_set_n(9, Q, c, x0, &tu, delta);
            }
            double qd[9];
            matvec(9, Q, delta, qd);
            const double quad = dotn(9, delta, qd);
            const double lin = 2.0 * dotn(9, c, delta);
            const double brier = (quad + lin) + 1.0;
            double g[9];
            for (int i = 0; i < 9; i++) g[i] = qd[i] + c[i];
            kor_output *o = &out[row0 + (y - x)];
            o->x = (uint64_t)x;
            o->y = (uint64_t)y;
            memcpy(o->jacquard, delta, sizeof delta);
            o->obj = brier;
            o->iters = its;
            o->cond = condition_estimate(delta, g, Q, tu.sqp_conv_tol);
        }
    }
    *n_out = npairs;
    free(site); free(p); free(q); free(msite); free(mf);
    return KOR_OK;
}

/* ---------------------------------- soft genotype likelihoods (the GL/PL path) */
/* The reference's GL/PL estimator on likelihoods that need not be one-hot
 * (src/wrapper.rs:89-330, src/allele/mod.rs, src/mixture.rs, src/coefficients.rs:
 * 40-141).  Likelihoods are linear-scale, genotype-major per sample in the VCF
 * order (G = 3, 6, 10 for 2, 3, 4 alleles); a sample whose row holds a NaN is
 * missing (src/vcf.rs:355, src/lanevector.rs:99-104 drop such rows). */

typedef struct {
    const double *gl;  /* n_samples x g */
    int64_t n_samples;
    int a, g;
    const double *w;   /* NULL, or a weight per row (rows standing for that many samples) */
} af_site_t;

static int row_ok(const double *r, int g) {
    for (int k = 0; k < g; k++)
        if (isnan(r[k])) return 0;
    return 1;
}

/* -(1/n) sum over called samples of log(eps + x' L x), L the symmetric matrix of
 * the sample's likelihoods (L_ii = GL(i,i), L_ij = L_ji = GL(i,j)): the HWE
 * mixture x_i^2 GL(i,i) + 2 x_i x_j GL(i,j) (src/allele/objective.rs). */
static double af_objective(const void *ctx, const double *x, double eps) {
    const af_site_t *s = (const af_site_t *)ctx;
    double acc = 0.0;
    int64_t n = 0;
    for (int64_t k = 0; k < s->n_samples; k++) {
        const double *r = s->gl + k * s->g;
        if (!row_ok(r, s->g)) continue;
        double p = eps;
        for (int b = 0; b < s->a; b++)
            for (int a = 0; a <= b; a++) {
                const double w = a == b ? x[a] * x[a] : 2.0 * x[a] * x[b];
                p = fma(w, r[b * (b + 1) / 2 + a], p);
            }
        const double wk = s->w ? s->w[k] : 1.0;
        acc = fma(wk, log(p), acc);
        n += (int64_t)wk;
    }
    return -acc / (double)n;
}

/* gradient -2/n sum Lx/d and Hessian 2/n sum (2 (Lx/d)(Lx/d)' - L/d), d =
 * eps + x' L x (src/allele/grad_hess.rs:81-172). */
static void af_grad_hess(const void *ctx, const double *x, double eps, double g[9], double H[9][9]) {
    const af_site_t *s = (const af_site_t *)ctx;
    const int A = s->a;
    double zg[4] = {0, 0, 0, 0}, zh[4][4];
    memset(zh, 0, sizeof zh);
    int64_t n = 0;
    for (int64_t k = 0; k < s->n_samples; k++) {
        const double *r = s->gl + k * s->g;
        if (!row_ok(r, s->g)) continue;
        double L[4][4];
        for (int b = 0; b < A; b++)
            for (int a = 0; a <= b; a++) L[a][b] = L[b][a] = r[b * (b + 1) / 2 + a];
        double lx[4], d = eps;
        for (int a = 0; a < A; a++) {
            lx[a] = 0.0;
            for (int b = 0; b < A; b++) lx[a] = fma(L[a][b], x[b], lx[a]);
        }
        for (int a = 0; a < A; a++) d = fma(x[a], lx[a], d);
        const double inv = 1.0 / d;
        const double wk = s->w ? s->w[k] : 1.0;
        for (int a = 0; a < A; a++) {
            zg[a] = fma(wk, lx[a] * inv, zg[a]);
            for (int b = 0; b < A; b++) zh[a][b] = fma(wk, 2.0 * (lx[a] * inv) * (lx[b] * inv) - L[a][b] * inv, zh[a][b]);
        }
        n += (int64_t)wk;
    }
    for (int i = 0; i < 9; i++) {
        g[i] = 0.0;
        for (int j = 0; j < 9; j++) H[i][j] = 0.0;
    }
    for (int a = 0; a < A; a++) {
        g[a] = -2.0 * zg[a] / (double)n;
        for (int b = 0; b < A; b++) H[a][b] = 2.0 * zh[a][b] / (double)n;
    }
}

static int kkt_converged_n(int n, const double *x, const double *g, double tol) {
    const double lambda = dotn(n, x, g);
    for (int i = 0; i < n; i++) {
        if (x[i] == 0.0) {
            if (!(g[i] >= lambda - tol)) return 0;
        } else if (!(fabs(g[i] - lambda) <= tol)) {
            return 0;
        }
    }
    return 1;
}

typedef double (*sqp_obj_fn)(const void *, const double *, double);
typedef void (*sqp_gh_fn)(const void *, const double *, double, double g[9], double H[9][9]);

/* src/sqp.rs:49-93 and :270-310 for a problem of dimension n <= 9 given by its
 * objective and gradient/Hessian; returns the iteration count. */
static uint64_t solve_sqp_n(int n, sqp_obj_fn fo, sqp_gh_fn fgh, const void *ctx, const double *x0,
                            const tune_t *tu, double x_out[9], double *f_out) {
    double x[9] = {0};
    sum_to_one_n(n, x0, x);
    double f = fo(ctx, x, tu->epsilon);
    for (uint64_t it = 0; it < tu->sqp_max_iter; it++) {
        double g[9], H[9][9];
        fgh(ctx, x, tu->epsilon, g, H);
        if (kkt_converged_n(n, x, g, tu->sqp_conv_tol)) {
            memcpy(x_out, x, sizeof x);
            *f_out = f;
            return it;
        }
        double hx[9] = {0}, c[9] = {0}, y[9] = {0}, p[9] = {0};
        matvec(n, H, x, hx);
        for (int i = 0; i < n; i++) c[i] = g[i] - hx[i];
        qp_active_set_n(n, H, c, x, tu, y);
        for (int i = 0; i < n; i++) p[i] = y[i] - x[i];
        const double t = tu->bls_sufficient_decrease * dotn(n, g, p);
        double alpha = 1.0, xs[9] = {0}, fn;
        uint64_t ls = 0;
        for (;;) {
            double xn[9] = {0};
            for (int i = 0; i < n; i++) xn[i] = x[i] + alpha * p[i];
            sum_to_one_n(n, xn, xs);
            fn = fo(ctx, xs, tu->epsilon);
            if (fn <= f + alpha * t) break;
            if (++ls == tu->bls_max_iter) break;
            alpha *= tu->bls_step_size_reduce;
        }
        memcpy(x, xs, sizeof x);
        f = fn;
    }
    memcpy(x_out, x, sizeof x);
    *f_out = f;
    return tu->sqp_max_iter;
}

/* One site's allele frequencies (src/allele/mod.rs:91-134): the SQP from 1/A
 * (sqp_max_iter = iterations, the QP at most A + 1 iterations); frequencies in
 * (0, maf) become 0 and the rest sum to one.  NaN when no sample is called. */
static void af_fit(const af_site_t *s, uint64_t iterations, double maf, double f_out[4]) {
    for (int a = 0; a < 4; a++) f_out[a] = 0.0;
    int64_t called = 0;
    for (int64_t k = 0; k < s->n_samples && !called; k++) called += row_ok(s->gl + k * s->g, s->g);
    if (!called) {
        for (int a = 0; a < s->a; a++) f_out[a] = NAN;
        return;
    }
    tune_t tu = make_tune(iterations);
    tu.qp_max_iter = (uint64_t)s->a + 1;
    double x0[9] = {0}, x[9], f;
    for (int a = 0; a < s->a; a++) x0[a] = 1.0 / s->a;
    solve_sqp_n(s->a, af_objective, af_grad_hess, s, x0, &tu, x, &f);
    for (int a = 0; a < s->a; a++)
        if (x[a] > 0.0 && x[a] < maf) x[a] = 0.0;
    sum_to_one_n(s->a, x, f_out);
}

static void hard_call_frequencies(const int64_t cnt[3], uint64_t iterations, double maf, double f[4]) {
    static const double one_hot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double rows[9], w[3];
    int n = 0;
    for (int c = 0; c < 3; c++)
        if (cnt[c] > 0) {
            memcpy(rows + 3 * n, one_hot + 3 * c, sizeof(double) * 3);
            w[n++] = (double)cnt[c];
        }
    af_site_t s = {rows, n, 2, 3, w};
    af_fit(&s, iterations, maf, f);
}

int kor_gl_allele_frequencies(const double *gl, int64_t n_sites, int64_t n_samples, int n_alleles,
                              uint64_t iterations, double maf, int threads, double *af_out) {
    if (!gl || !af_out || n_sites < 0 || n_samples <= 0 || n_alleles < 2 || n_alleles > 4 || iterations == 0)
        return KOR_EINVAL;
    const int g = n_alleles * (n_alleles + 1) / 2;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
#endif
    for (int64_t v = 0; v < n_sites; v++) {
        af_site_t s = {gl + v * n_samples * g, n_samples, n_alleles, g, NULL};
        af_fit(&s, iterations, maf, af_out + 4 * v);
    }
    return KOR_OK;
}

/* A site after its zero-frequency alleles are dropped (src/wrapper.rs:349-409):
 * the kept alleles (in order), their frequencies, for each kept genotype its
 * index in the original VCF order, and m[gx][gy] over the kept genotypes. */
typedef struct {
    const double *gl;  /* the original n_samples x g0 likelihoods */
    int g0, a, g;
    int gidx[10];
    double *m;         /* g x g x 9 */
} red_site_t;

int kor_gl_relatedness(const double *gl2, int64_t n2, const double *gl3, int64_t n3, const double *gl4,
                       int64_t n4, int64_t n_samples, double maf, int64_t num_samples, uint64_t iterations,
                       int threads, kor_output *out, int64_t out_cap, int64_t *n_out, double *af_out) {
    if (n_samples <= 0 || n2 < 0 || n3 < 0 || n4 < 0 || (n2 && !gl2) || (n3 && !gl3) || (n4 && !gl4) || !out ||
        !n_out || iterations == 0)
        return KOR_EINVAL;
    if (num_samples < 0) num_samples = n_samples;
    if (num_samples == 0 || num_samples > n_samples) return KOR_EINVAL;
    const int64_t npairs = num_samples * (num_samples + 1) / 2;
    if (out_cap < npairs) return KOR_EINVAL;
    if (!(maf >= 0.0)) maf = 1.0 / (2.0 * (double)n_samples);   /* src/wrapper.rs:99-101 */
    const int64_t nv = n2 + n3 + n4;
    const double *gls[3] = {gl2, gl3, gl4};
    const int64_t ns[3] = {n2, n3, n4};
    double *af = (double *)malloc(sizeof(double) * 4 * (size_t)(nv + 1));
    red_site_t *lists[3];
    int64_t counts[3] = {0, 0, 0};
    for (int k = 0; k < 3; k++) lists[k] = (red_site_t *)calloc((size_t)(nv + 1), sizeof(red_site_t));
    if (!af || !lists[0] || !lists[1] || !lists[2]) {
        free(af); free(lists[0]); free(lists[1]); free(lists[2]);
        return KOR_ENOMEM;
    }
    /* frequencies of every site, bi-, tri- then tetra-allelic */
    int64_t off = 0;
    for (int k = 0; k < 3; k++) {
        kor_gl_allele_frequencies(gls[k], ns[k], n_samples, k + 2, iterations, maf, threads, af + 4 * off);
        off += ns[k];
    }
    if (af_out) memcpy(af_out, af, sizeof(double) * 4 * (size_t)nv);
    /* drop zero-frequency alleles, in the reference's order: each group's sites
     * go to the list of their remaining allele count */
    off = 0;
    for (int k = 0; k < 3; k++) {
        const int a0 = k + 2, g0 = a0 * (a0 + 1) / 2;
        for (int64_t v = 0; v < ns[k]; v++) {
            const double *f = af + 4 * (off + v);
            int keep[4], na = 0;
            double fk[4] = {0, 0, 0, 0};
            for (int a = 0; a < a0; a++)
                if (f[a] > 0.0) { keep[na] = a; fk[na] = f[a]; na++; }
            if (na < 2) continue;
            red_site_t *r = &lists[na - 2][counts[na - 2]++];
            r->gl = gls[k] + v * n_samples * g0;
            r->g0 = g0;
            r->a = na;
            r->g = na * (na + 1) / 2;
            int t = 0;
            for (int j = 0; j < na; j++)
                for (int i = 0; i <= j; i++) r->gidx[t++] = keep[j] * (keep[j] + 1) / 2 + keep[i];
            r->m = (double *)malloc(sizeof(double) * 9 * (size_t)(r->g * r->g));
            if (r->m)
                for (int gx = 0; gx < r->g; gx++)
                    for (int gy = 0; gy < r->g; gy++) kor_iis_row(gx, gy, fk, r->m + 9 * (gx * r->g + gy));
        }
        off += ns[k];
    }
    const int64_t nk = counts[0] + counts[1] + counts[2];
    int st = nk == 0 ? KOR_ENOSITES : KOR_OK;
    for (int k = 0; k < 3 && st == KOR_OK; k++)
        for (int64_t v = 0; v < counts[k]; v++)
            if (!lists[k][v].m) st = KOR_ENOMEM;
    if (st == KOR_OK) {
        tune_t tu = make_tune(iterations);
#ifdef _OPENMP
        if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
#endif
        {
            rowbuf_t rb;
            rb.blocks = (v8d *)aligned_alloc(64, sizeof(v8d) * 9 * (size_t)(nk / 8 + 1));
            pass_count_t pc = {0, 0};
            if (rb.blocks) {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
                for (int64_t x = 0; x < num_samples; x++) {
                    const int64_t row0 = x * num_samples - x * (x - 1) / 2;
                    for (int64_t y = x; y < num_samples; y++) {
                        rb_reset(&rb);
                        /* the pair's rows: sum over genotype pairs of GLx GLy m
                         * (src/mixture.rs:9-62), bi-, tri- then tetra-allelic */
                        for (int k = 0; k < 3; k++)
                            for (int64_t v = 0; v < counts[k]; v++) {
                                const red_site_t *r = &lists[k][v];
                                const double *lx = r->gl + x * r->g0, *ly = r->gl + y * r->g0;
                                double row[9] = {0};
                                for (int gx = 0; gx < r->g; gx++) {
                                    const double ax = lx[r->gidx[gx]];
                                    for (int gy = 0; gy < r->g; gy++) {
                                        const double gg = ax * ly[r->gidx[gy]];
                                        const double *mm = r->m + 9 * (gx * r->g + gy);
                                        for (int s = 0; s < 9; s++) row[s] = fma(gg, mm[s], row[s]);
                                    }
                                }
                                if (row_ok(row, 9)) rb_push(&rb, row);
                            }
                        rb_finish(&rb);
                        kor_output *o = out + row0 + (y - x);
                        o->x = (uint64_t)x;
                        o->y = (uint64_t)y;
                        if (rb_len(&rb) == 0) {
                            memset(o->jacquard, 0, sizeof o->jacquard);
                            o->obj = NAN; o->iters = 0; o->cond = NAN;
                            continue;
                        }
                        double x0[9] = {0};
                        if (x == y) { x0[0] = 0.5; x0[6] = 0.5; }
                        else for (int i = 0; i < 9; i++) x0[i] = 1.0 / 9.0;
                        solve_sqp(&rb, x0, &tu, o, &pc);
                    }
                }
                free(rb.blocks);
            }
        }
        *n_out = npairs;
    }
    for (int k = 0; k < 3; k++) {
        for (int64_t v = 0; v < counts[k]; v++) free(lists[k][v].m);
        free(lists[k]);
    }
    free(af);
    return st;
}
