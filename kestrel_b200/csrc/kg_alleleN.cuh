// kg_alleleN.cuh — the allele-frequency fit of a site with up to four alleles
// from its hard calls, as the reference's GL/PL path computes it on one-hot
// likelihoods (src/allele/mod.rs:91-134 with src/allele/objective.rs and
// src/allele/grad_hess.rs): the SQP of src/sqp.rs:49-93 on the A-dimensional
// simplex from 1/A, at most `iterations` iterations, the QP of
// src/sqp.rs:112-250 at most A + 1 iterations, the GMW81-modified LDL^T of
// src/cholesky.rs:6-65 and its solves (:104-140); then frequencies in (0, maf)
// become zero and the rest are renormalised.
//
// The sums run over weighted likelihood rows (genotype g = j (j + 1) / 2 + i
// for alleles i <= j, the VCF order), given by a row source: with one-hot
// likelihoods the objective -(1/n) sum_samples log(eps + x'Lx) only depends on
// how many samples carry each genotype, so AlleleClasses gives the site's
// genotype classes, each weighted by its count; soft likelihoods give one row
// per called sample.  One thread per site: every array is at most 4 or 4 x 4.
#pragma once

#include <cstdint>

#include "kg_solver.cuh"

namespace kg {

constexpr int MAXA = 4;    // alleles
constexpr int MAXG = 10;   // genotypes of four alleles

struct AlleleClasses {
    int a;               // alleles (2..4)
    int n;               // classes with a non-zero count
    int cls[MAXG];       // their genotype indices
    double w[MAXG];      // their counts
    // the row source: row k's likelihoods (one-hot at its genotype) and weight
    __host__ __device__ int alleles() const { return a; }
    __host__ __device__ int rows() const { return n; }
    __host__ __device__ double weight(int k) const { return w[k]; }
    __host__ __device__ bool row(int k, double* l) const {
        for (int g = 0; g < MAXG; g++) l[g] = g == cls[k] ? 1.0 : 0.0;
        return true;
    }
};

// The likelihood matrix entry L[r][c] of a row l (L symmetric: L[i][j] =
// L[j][i] = l[genotype (i, j)]).
__host__ __device__ __forceinline__ double lmat(const double* l, int r, int c) {
    const int i = r < c ? r : c, j = r < c ? c : r;
    return l[j * (j + 1) / 2 + i];
}

// -(1/n) sum over rows of weight x log(eps + sum over genotypes (a <= b) of
// w_ab L_ab), w_aa = x_a^2, w_ab = 2 x_a x_b, fused in the reference's order
// (src/allele/objective.rs); rows with a NaN are skipped.
template <class Src>
__host__ __device__ inline double allele_objective(const Src& C, const double* x, double eps) {
    double acc = 0.0, tot = 0.0;
    const int A = C.alleles();
    for (int k = 0; k < C.rows(); k++) {
        double l[MAXG];
        if (!C.row(k, l)) continue;
        double p = eps;
        for (int b = 0; b < A; b++)
            for (int a = 0; a <= b; a++) {
                const double w = a == b ? x[a] * x[a] : 2.0 * x[a] * x[b];
                p = fma(w, l[b * (b + 1) / 2 + a], p);
            }
        acc = fma(C.weight(k), log(p), acc);
        tot += C.weight(k);
    }
    return -acc / tot;
}

// gradient -2/n sum Lx/d and Hessian 2/n sum (2 (Lx/d)(Lx/d)' - L/d), d = eps
// + x'Lx (src/allele/grad_hess.rs), per row weighted.
template <class Src>
__host__ __device__ inline void allele_grad_hess(const Src& C, const double* x, double eps, double* g,
                                                 double (*H)[MAXA]) {
    const int A = C.alleles();
    double zg[MAXA], zh[MAXA][MAXA], tot = 0.0;
    for (int a = 0; a < MAXA; a++) {
        zg[a] = 0.0;
        for (int b = 0; b < MAXA; b++) zh[a][b] = 0.0;
    }
    for (int k = 0; k < C.rows(); k++) {
        double l[MAXG];
        if (!C.row(k, l)) continue;
        const double wk = C.weight(k);
        double lx[MAXA], d = eps;
        for (int a = 0; a < A; a++) {
            lx[a] = 0.0;
            for (int b = 0; b < A; b++) lx[a] = fma(lmat(l, a, b), x[b], lx[a]);
        }
        for (int a = 0; a < A; a++) d = fma(x[a], lx[a], d);
        const double inv = 1.0 / d;
        for (int a = 0; a < A; a++) {
            zg[a] = fma(wk, lx[a] * inv, zg[a]);
            for (int b = 0; b < A; b++)
                zh[a][b] = fma(wk, 2.0 * (lx[a] * inv) * (lx[b] * inv) - lmat(l, a, b) * inv, zh[a][b]);
        }
        tot += wk;
    }
    for (int a = 0; a < MAXA; a++) {
        g[a] = a < A ? -2.0 * zg[a] / tot : 0.0;
        for (int b = 0; b < MAXA; b++) H[a][b] = (a < A && b < A) ? 2.0 * zh[a][b] / tot : 0.0;
    }
}

__host__ __device__ __forceinline__ double dotn4(int n, const double* a, const double* b) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s = fma(a[i], b[i], s);
    return s;
}

__host__ __device__ __forceinline__ double sumn4(int n, const double* a) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i];
    return s;
}

// GMW81-modified LDL^T of the leading n x n block (src/cholesky.rs:6-65).
__host__ __device__ inline void gmw_ldl4(int n, const double (*a)[MAXA], double (*l)[MAXA], double* d) {
    double gamma = 0.0, xi = 0.0;
    for (int i = 0; i < n; i++) gamma = fmax(gamma, fabs(a[i][i]));
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) xi = fmax(xi, fabs(a[i][j]));
    const double eps = 2.220446049250313e-16;
    const double delta = eps * fmax(1.0, gamma + xi);
    const double t = sqrt((double)n * (double)n - 1.0);
    const double ratio = n <= 1 ? 0.0 : xi / t;
    const double beta2 = fmax(fmax(gamma, ratio), eps);
    double pv[MAXA];
    for (int j = 0; j < n; j++) {
        double sjj = 0.0;
        for (int s = 0; s < j; s++) {
            pv[s] = d[s] * l[j][s];
            sjj = fma(pv[s], l[j][s], sjj);
        }
        const double cjj = a[j][j] - sjj;
        l[j][j] = 1.0;
        double theta = 0.0;
        for (int i = j + 1; i < n; i++) {
            double sij = 0.0;
            for (int s = 0; s < j; s++) sij = fma(pv[s], l[i][s], sij);
            const double cij = a[i][j] - sij;
            theta = fmax(theta, fabs(cij));
            l[i][j] = cij;
        }
        const double dj = fmax(fmax(fabs(cjj), theta * theta / beta2), delta);
        for (int i = j + 1; i < n; i++) l[i][j] /= dj;
        d[j] = dj;
    }
}

// L D L^T z = b in place (src/cholesky.rs:104-140).
__host__ __device__ inline void ldl_solve4(int n, const double (*l)[MAXA], const double* d, double* b) {
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = 0; j < i; j++) s = fma(b[j], l[i][j], s);
        b[i] -= s;
    }
    for (int i = 0; i < n; i++) b[i] /= d[i];
    for (int i = n - 1; i >= 0; i--) {
        double s = 0.0;
        for (int j = i + 1; j < n; j++) s = fma(b[j], l[j][i], s);
        b[i] -= s;
    }
}

// min 1/2 y'Qy + c'y on the n-simplex from y0 by the active-set method of
// src/sqp.rs:112-250 (modify = true), at most qp_max_iter iterations.
__host__ __device__ inline void qp_simplex4(int n, const double (*Q)[MAXA], const double* c, const double* y0,
                                            int qp_max_iter, const Tune& tq, double* y) {
    bool work[MAXA];
    for (int i = 0; i < MAXA; i++) {
        y[i] = i < n ? y0[i] : 0.0;
        work[i] = i < n && y[i] == 0.0;
    }
    for (int it = 0; it < qp_max_iter; it++) {
        const double sy = sumn4(n, y);
        for (int i = 0; i < n; i++) y[i] = y[i] / sy;
        int fi[MAXA], nf = 0;
        for (int i = 0; i < n; i++)
            if (!work[i]) fi[nf++] = i;
        if (nf == 0) return;   // the reference asserts this cannot happen
        double yf[MAXA], gf[MAXA], Qf[MAXA][MAXA], L[MAXA][MAXA], D[MAXA], ones[MAXA];
        for (int i = 0; i < MAXA; i++) {
            yf[i] = i < nf ? y[fi[i]] : 0.0;
            D[i] = 0.0;
            ones[i] = i < nf ? 1.0 : 0.0;
            for (int j = 0; j < MAXA; j++) {
                Qf[i][j] = (i < nf && j < nf) ? Q[fi[i]][fi[j]] : 0.0;
                L[i][j] = 0.0;
            }
        }
        for (int i = 0; i < nf; i++) gf[i] = c[fi[i]] + dotn4(nf, Qf[i], yf);
        for (int i = nf; i < MAXA; i++) gf[i] = 0.0;
        gmw_ldl4(nf, Qf, L, D);
        ldl_solve4(nf, L, D, gf);
        ldl_solve4(nf, L, D, ones);
        const double lambda = sumn4(nf, gf) / sumn4(nf, ones);
        // lambda * ones - g over all slots (those past nf are zero on both
        // sides); the largest magnitude, NaN ranking highest
        double m = 0.0;
        bool m_nan = false;
        for (int i = 0; i < n; i++) {
            gf[i] = lambda * ones[i] - gf[i];
            const double a = fabs(gf[i]);
            if (isnan(a)) m_nan = true;
            else if (a > m) m = a;
        }
        if (!m_nan && m <= tq.qp_zero_search_tol) {
            if (nf == n) return;
            double gq[MAXA];
            for (int i = 0; i < n; i++) gq[i] = c[i] + dotn4(n, Q[i], y);
            int best = -1;
            for (int i = 0; i < n; i++)
                if (work[i] && (best < 0 || gq[i] < gq[best])) best = i;
            if (gq[best] - lambda >= -tq.qp_conv_tol) return;
            work[best] = false;
        } else {
            double p[MAXA];
            int k = 0;
            for (int i = 0; i < n; i++) p[i] = work[i] ? 0.0 : gf[k++];
            double alpha = 1.0;
            int block = -1;
            for (int i = 0; i < n; i++)
                if (p[i] < 0.0) {
                    const double a = -y[i] / p[i];
                    if (a < alpha) { alpha = a; block = i; }
                }
            for (int i = 0; i < n; i++) y[i] = fmax(y[i] + alpha * p[i], 0.0);
            if (block >= 0) { work[block] = true; y[block] = 0.0; }
        }
    }
}

// The fit of one site: f gets its A frequencies (zero past A).  A site
// without a called row gets NaN frequencies (its sums have no term).
template <class Src>
__host__ __device__ inline void allele_fit(const Src& C, uint64_t iterations, double maf, double* f) {
    const int A = C.alleles();
    for (int a = 0; a < MAXA; a++) f[a] = 0.0;
    bool any = false;
    for (int k = 0; k < C.rows() && !any; k++) {
        double l[MAXG];
        any = C.row(k, l);
    }
    if (!any) {
        for (int a = 0; a < A; a++) f[a] = nan("");
        return;
    }
    const Tune tq = make_tune(iterations);
    const int qp_iters = A + 1;   // src/allele/mod.rs:100
    double x[MAXA], x0[MAXA];
    for (int a = 0; a < MAXA; a++) x0[a] = a < A ? 1.0 / A : 0.0;
    const double s0 = sumn4(A, x0);
    for (int a = 0; a < MAXA; a++) x[a] = a < A ? x0[a] / s0 : 0.0;
    double fx = allele_objective(C, x, tq.epsilon);
    for (uint64_t it = 0; it < iterations; it++) {
        double g[MAXA], H[MAXA][MAXA];
        allele_grad_hess(C, x, tq.epsilon, g, H);
        // KKT on the simplex (src/sqp.rs:95-109)
        const double lambda = dotn4(A, x, g);
        bool ok = true;
        for (int a = 0; a < A; a++)
            ok = ok && (x[a] == 0.0 ? (g[a] >= lambda - tq.sqp_conv_tol) : (fabs(g[a] - lambda) <= tq.sqp_conv_tol));
        if (ok) break;
        double c[MAXA], y[MAXA], p[MAXA];
        for (int a = 0; a < A; a++) c[a] = g[a] - dotn4(A, H[a], x);
        qp_simplex4(A, H, c, x, qp_iters, tq, y);
        for (int a = 0; a < A; a++) p[a] = y[a] - x[a];
        const double t = tq.bls_sufficient_decrease * dotn4(A, g, p);
        double alpha = 1.0, xs[MAXA], fn;
        for (int ls = 0;;) {
            double xn[MAXA];
            for (int a = 0; a < A; a++) xn[a] = x[a] + alpha * p[a];
            const double sn = sumn4(A, xn);
            for (int a = 0; a < A; a++) xs[a] = xn[a] / sn;
            fn = allele_objective(C, xs, tq.epsilon);
            if (fn <= fx + alpha * t) break;
            if (++ls == tq.bls_max_iter) break;
            alpha *= tq.bls_step_size_reduce;
        }
        for (int a = 0; a < A; a++) x[a] = xs[a];
        fx = fn;
    }
    for (int a = 0; a < A; a++)
        if (x[a] > 0.0 && x[a] < maf) x[a] = 0.0;
    const double s = sumn4(A, x);
    for (int a = 0; a < A; a++) f[a] = x[a] / s;
}

}  // namespace kg
