// kg_solver.cuh — FP64 9-variable SQP pieces run by one warp per pair.
//
// Every lane of the warp executes the same scalar code on identical data, so
// the results are warp-uniform without broadcasts; the arrays live in each
// lane's local memory (L1-cached).  The algorithm is the reference's, restated:
//   check_convergence        src/sqp.rs:95-109
//   estimate_condition_number src/sqp.rs:313-391
//   unmodified_n / forward and back substitution  src/cholesky.rs:66-140
//   dot (fma chain), sum_to_one  src/algebra.rs:4-84
// The QP and its GMW81-modified LDL^T run row-parallel (kg_rowsolve.cuh).
#pragma once

#include <math_constants.h>

#include <cstdint>
#include <cmath>

namespace kg {

struct Tune {
    uint64_t sqp_max_iter;
    double sqp_conv_tol;        // 1e-8
    int qp_max_iter;            // 10 on the ML path (src/coefficients.rs:73)
    double qp_conv_tol;         // 1e-10
    double qp_zero_search_tol;  // 1e-12
    int bls_max_iter;           // 10
    double bls_sufficient_decrease;  // 1e-4
    double bls_step_size_reduce;     // 0.9
    double epsilon;             // 1e-8
};

__host__ __device__ inline Tune make_tune(uint64_t iters) {
    Tune t;
    t.sqp_max_iter = iters;
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

__device__ __forceinline__ double dot_fma(int n, const double* a, const double* b) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s = fma(a[i], b[i], s);
    return s;
}

__device__ __forceinline__ double sum_seq(int n, const double* a) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i];
    return s;
}

__device__ __forceinline__ void normalise9(double* x) {
    double s = sum_seq(9, x);
    for (int i = 0; i < 9; i++) x[i] = x[i] / s;
}

// KKT test on the simplex; *resid gets the largest violation (for the FP32 ->
// FP64 escalation rule).
__device__ inline bool kkt_ok(const double* x, const double* g, double tol, double* resid) {
    double lambda = dot_fma(9, x, g);
    bool ok = true;
    double r = 0.0;
    for (int i = 0; i < 9; i++) {
        double v;
        if (x[i] == 0.0) {
            ok = ok && (g[i] >= lambda - tol);
            v = lambda - g[i];
        } else {
            double a = fabs(g[i] - lambda);
            ok = ok && (a <= tol);
            v = a;
        }
        r = fmax(r, v);
    }
    *resid = r;
    return ok;
}


// Plain LDL^T (no pivoting, no modification).
__device__ inline void ldl_plain(int n, const double* a, double* l, double* d) {
    double pv[9];
    for (int j = 0; j < n; j++) {
        l[j * 9 + j] = 1.0;
        double sjj = 0.0;
        for (int s = 0; s < j; s++) {
            pv[s] = d[s] * l[j * 9 + s];
            sjj = fma(pv[s], l[j * 9 + s], sjj);
        }
        double dj = a[j * 9 + j] - sjj;
        for (int i = j + 1; i < n; i++) {
            double sij = 0.0;
            for (int s = 0; s < j; s++) sij = fma(pv[s], l[i * 9 + s], sij);
            l[i * 9 + j] = (a[i * 9 + j] - sij) / dj;
        }
        d[j] = dj;
    }
}

__device__ __forceinline__ void unit_lower_solve(int n, const double* l, double* b) {
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = 0; j < i; j++) s = fma(b[j], l[i * 9 + j], s);
        b[i] -= s;
    }
}

__device__ __forceinline__ void unit_upper_solve_t(int n, const double* l, double* b) {
    for (int i = n - 1; i >= 0; i--) {
        double s = 0.0;
        for (int j = i + 1; j < n; j++) s = fma(b[j], l[j * 9 + i], s);
        b[i] -= s;
    }
}



// Condition estimate of the reduced Hessian at a KKT point.
__device__ inline double condition_estimate(const double* x, const double* g, const double* H,
                                            double tol) {
    double lambda = dot_fma(9, x, g);
    int fi[9];
    int nf = 0;
    for (int i = 0; i < 9; i++) {
        bool strict = (x[i] == 0.0) && (g[i] >= lambda + tol);
        if (!strict) fi[nf++] = i;
    }
    if (nf == 0) return CUDART_INF;
    double Hf[81], L[81], D[9];
    for (int i = 0; i < 81; i++) { Hf[i] = 0.0; L[i] = 0.0; }
    for (int i = 0; i < 9; i++) D[i] = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) Hf[i * 9 + j] = H[fi[i] * 9 + fi[j]];
    ldl_plain(nf, Hf, L, D);
    for (int i = 0; i < nf; i++)
        if (!(D[i] > 0.0)) return CUDART_INF;
    int imax = 0, imin = 0;
    for (int i = 1; i < nf; i++) {
        if (D[i] >= D[imax]) imax = i;
        if (D[i] < D[imin]) imin = i;
    }
    double emax[9], emin[9], w[9];
    for (int i = 0; i < 9; i++) { emax[i] = 0.0; emin[i] = 0.0; }
    emax[imax] = 1.0;
    emin[imin] = 1.0;
    for (int i = 0; i < nf; i++) w[i] = dot_fma(nf, L + i * 9, emax);
    unit_upper_solve_t(nf, L, emin);
    double nmax = sqrt(dot_fma(nf, w, w));
    double nmin = sqrt(dot_fma(nf, emin, emin));
    return nmax * nmin * (D[imax] / D[imin]);
}

// The active-set QP of src/sqp.rs:112-250 on the two-dimensional simplex from
// (s0, s1), written out on scalars (GMW81 LDL^T of src/cholesky.rs:6-65 for one
// or two free variables): the CLS self pairs' (Delta1, Delta7) step and the
// biallelic allele-frequency fit.  Returns the iteration count.
__host__ __device__ inline int qp_simplex2(double q00, double q01, double q10, double q11, double c0, double c1,
                                           double s0, double s1, const Tune& tq, double& y0, double& y1) {
    const double eps = 2.220446049250313e-16;
    y0 = s0;
    y1 = s1;
    bool w0 = y0 == 0.0, w1 = y1 == 0.0;
    int it = 0;
    while (it < tq.qp_max_iter) {
        const double sy = (0.0 + y0) + y1;
        y0 = y0 / sy;
        y1 = y1 / sy;
        const int nf = (w0 ? 0 : 1) + (w1 ? 0 : 1);
        if (nf == 0) return it;
        double lambda, p0 = 0.0, p1 = 0.0, m;
        bool m_nan;
        if (nf == 2) {
            const double g0 = c0 + fma(q01, y1, fma(q00, y0, 0.0));
            const double g1 = c1 + fma(q11, y1, fma(q10, y0, 0.0));
            const double gamma = fmax(fmax(0.0, fabs(q00)), fabs(q11));
            const double xi = fmax(0.0, fabs(q01));
            const double delta = eps * fmax(1.0, gamma + xi);
            const double beta2 = fmax(fmax(gamma, xi / sqrt(3.0)), eps);
            const double theta = fmax(0.0, fabs(q10));
            const double d0 = fmax(fmax(fabs(q00), theta * theta / beta2), delta);
            const double l10 = q10 / d0;
            const double pv0 = d0 * l10;
            const double d1 = fmax(fmax(fabs(q11 - fma(pv0, l10, 0.0)), 0.0 / beta2), delta);
            double b0 = g0, b1 = g1 - fma(b0, l10, 0.0);
            b0 = b0 / d0;
            b1 = b1 / d1;
            b0 = b0 - fma(b1, l10, 0.0);
            double o0 = 1.0, o1 = 1.0 - fma(o0, l10, 0.0);
            o0 = o0 / d0;
            o1 = o1 / d1;
            o0 = o0 - fma(o1, l10, 0.0);
            lambda = ((0.0 + b0) + b1) / ((0.0 + o0) + o1);
            const double f0 = lambda * o0 - b0, f1 = lambda * o1 - b1;
            m_nan = isnan(f0) || isnan(f1);
            m = fmax(fabs(f0), fabs(f1));
            p0 = f0;
            p1 = f1;
        } else {
            // one free variable k: the 1 x 1 factor
            const bool k0 = !w0;
            const double a = k0 ? q00 : q11, ck = k0 ? c0 : c1, yk = k0 ? y0 : y1;
            const double g = ck + fma(a, yk, 0.0);
            const double gamma = fmax(0.0, fabs(a));
            const double delta = eps * fmax(1.0, gamma + 0.0);
            const double d0 = fmax(fmax(fabs(a), 0.0), delta);
            const double b = g / d0, o = 1.0 / d0;
            lambda = (0.0 + b) / (0.0 + o);
            const double f = lambda * o - b, f_pad = lambda * 0.0 - 0.0;
            m_nan = isnan(f) || isnan(f_pad);
            m = fmax(fabs(f), fabs(f_pad));
            if (k0) p0 = f;
            else p1 = f;
        }
        if (!m_nan && m <= tq.qp_zero_search_tol) {
            if (nf == 2) return it;
            const double gq0 = c0 + fma(q01, y1, fma(q00, y0, 0.0));
            const double gq1 = c1 + fma(q11, y1, fma(q10, y0, 0.0));
            const int best = w0 ? ((w1 && gq1 < gq0) ? 1 : 0) : 1;
            const double gb = best == 0 ? gq0 : gq1;
            if (gb - lambda >= -tq.qp_conv_tol) return it;
            if (best == 0) w0 = false;
            else w1 = false;
        } else {
            double alpha = 1.0;
            int block = -1;
            if (p0 < 0.0) {
                const double a = -y0 / p0;
                if (a < alpha) { alpha = a; block = 0; }
            }
            if (p1 < 0.0) {
                const double a = -y1 / p1;
                if (a < alpha) { alpha = a; block = 1; }
            }
            y0 = fmax(y0 + alpha * p0, 0.0);
            y1 = fmax(y1 + alpha * p1, 0.0);
            if (block == 0) { w0 = true; y0 = 0.0; }
            if (block == 1) { w1 = true; y1 = 0.0; }
        }
        it++;
    }
    return it;
}

}  // namespace kg
