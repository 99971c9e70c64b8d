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

}  // namespace kg
