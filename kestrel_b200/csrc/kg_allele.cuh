// kg_allele.cuh — the allele-frequency fit of a biallelic site from its hard
// calls, as the reference's GL/PL path computes it on one-hot likelihoods
// (src/allele/mod.rs:91-134, src/allele/objective.rs, src/allele/grad_hess.rs):
// the SQP of src/sqp.rs:49-93 on the two-dimensional simplex from (1/2, 1/2),
// with the iteration cap of the estimator and at most 3 QP iterations, then
// frequencies in (0, maf) set to zero and the rest renormalised.
//
// On one-hot likelihoods the objective -(1/n) sum log(eps + x'Lx) depends on
// the genotype-class counts only: n00 log(eps + x0^2) + n01 log(eps + 2 x0 x1)
// + n11 log(eps + x1^2).  The eps = 1e-8 inside the log puts the optimum about
// 5e-9 below the count frequency, so a count frequency equal to maf is cut.
#pragma once

#include <cstdint>

#include "kg_solver.cuh"

namespace kg {

// -(1/n) sum over classes of count x log(eps + x'Lx), classes in the order
// 0/0, 0/1, 1/1 (empty classes skipped); the mixture term as the reference
// forms it: eps plus the one-hot row's single product.
__host__ __device__ inline double allele2_objective(const double n[3], double x0, double x1, double eps) {
    double acc = 0.0, tot = 0.0;
    const double w[3] = {x0 * x0, 2.0 * x0 * x1, x1 * x1};
    for (int c = 0; c < 3; c++) {
        if (n[c] <= 0.0) continue;
        const double p = fma(w[c], 1.0, eps);
        acc = fma(n[c], log(p), acc);
        tot += n[c];
    }
    return -acc / tot;
}

// gradient -2/n sum Lx/d and Hessian 2/n sum (2 (Lx/d)(Lx/d)' - L/d), d =
// eps + x'Lx, per class (L the class's one-hot genotype matrix).
__host__ __device__ inline void allele2_grad_hess(const double n[3], double x0, double x1, double eps, double& g0,
                                                  double& g1, double& h00, double& h01, double& h11) {
    double zg0 = 0.0, zg1 = 0.0, z00 = 0.0, z01 = 0.0, z11 = 0.0, tot = 0.0;
    for (int c = 0; c < 3; c++) {
        if (n[c] <= 0.0) continue;
        // L: 0/0 -> [[1,0],[0,0]], 0/1 -> [[0,1],[1,0]], 1/1 -> [[0,0],[0,1]]
        const double l00 = c == 0 ? 1.0 : 0.0, l01 = c == 1 ? 1.0 : 0.0, l11 = c == 2 ? 1.0 : 0.0;
        const double lx0 = fma(l01, x1, fma(l00, x0, 0.0));
        const double lx1 = fma(l11, x1, fma(l01, x0, 0.0));
        const double d = fma(x1, lx1, fma(x0, lx0, eps));
        const double inv = 1.0 / d;
        const double a0 = lx0 * inv, a1 = lx1 * inv;
        zg0 = fma(n[c], a0, zg0);
        zg1 = fma(n[c], a1, zg1);
        z00 = fma(n[c], 2.0 * a0 * a0 - l00 * inv, z00);
        z01 = fma(n[c], 2.0 * a0 * a1 - l01 * inv, z01);
        z11 = fma(n[c], 2.0 * a1 * a1 - l11 * inv, z11);
        tot += n[c];
    }
    g0 = -2.0 * zg0 / tot;
    g1 = -2.0 * zg1 / tot;
    h00 = 2.0 * z00 / tot;
    h01 = 2.0 * z01 / tot;
    h11 = 2.0 * z11 / tot;
}

// The SQP of the fit on the two-dimensional simplex from (1/2, 1/2), given the
// objective obj(x0, x1) and gh(x0, x1, g0, g1, h00, h01, h11); then the maf
// cut and renormalisation.
template <class Obj, class GH>
__host__ __device__ inline void allele2_fit(const Obj& obj, const GH& gh, uint64_t iterations, double maf,
                                            double& p, double& q) {
    Tune tq = make_tune(iterations);
    tq.qp_max_iter = 3;   // A + 1 (src/allele/mod.rs:100)
    double x0 = 0.5 / (0.5 + 0.5), x1 = 0.5 / (0.5 + 0.5);
    double f = obj(x0, x1);
    for (uint64_t it = 0; it < iterations; it++) {
        double g0, g1, h00, h01, h11;
        gh(x0, x1, g0, g1, h00, h01, h11);
        // KKT of the simplex: lambda = x.g; free coordinates at lambda, zero
        // ones at or above it (src/sqp.rs:95-110)
        const double lambda = fma(x1, g1, fma(x0, g0, 0.0));
        const bool ok0 = x0 == 0.0 ? (g0 >= lambda - tq.sqp_conv_tol) : (fabs(g0 - lambda) <= tq.sqp_conv_tol);
        const bool ok1 = x1 == 0.0 ? (g1 >= lambda - tq.sqp_conv_tol) : (fabs(g1 - lambda) <= tq.sqp_conv_tol);
        if (ok0 && ok1) break;
        // c = g - H x, the QP from x
        const double c0 = g0 - fma(h01, x1, fma(h00, x0, 0.0));
        const double c1 = g1 - fma(h11, x1, fma(h01, x0, 0.0));
        double y0, y1;
        qp_simplex2(h00, h01, h01, h11, c0, c1, x0, x1, tq, y0, y1);
        // backtracking line search (src/sqp.rs:270-310)
        const double p0 = y0 - x0, p1 = y1 - x1;
        const double t = tq.bls_sufficient_decrease * fma(g1, p1, fma(g0, p0, 0.0));
        double alpha = 1.0, s0 = x0, s1 = x1, fn = f;
        for (int ls = 0;;) {
            const double xn0 = x0 + alpha * p0, xn1 = x1 + alpha * p1;
            const double sm = (0.0 + xn0) + xn1;
            s0 = xn0 / sm;
            s1 = xn1 / sm;
            fn = obj(s0, s1);
            if (fn <= f + alpha * t) break;
            if (++ls == tq.bls_max_iter) break;
            alpha *= tq.bls_step_size_reduce;
        }
        x0 = s0;
        x1 = s1;
        f = fn;
    }
    if (x0 > 0.0 && x0 < maf) x0 = 0.0;
    if (x1 > 0.0 && x1 < maf) x1 = 0.0;
    const double sm = (0.0 + x0) + x1;
    p = x0 / sm;
    q = x1 / sm;
}

// The frequencies (REF, ALT) of a site with class counts n00, n01, n11 (at
// least one call); iterations is the SQP cap.
__host__ __device__ inline void allele2_frequencies(double n00, double n01, double n11, uint64_t iterations,
                                                    double maf, double& p, double& q) {
    const double n[3] = {n00, n01, n11};
    const double eps = make_tune(iterations).epsilon;
    allele2_fit([&](double x0, double x1) { return allele2_objective(n, x0, x1, eps); },
                [&](double x0, double x1, double& g0, double& g1, double& h00, double& h01, double& h11) {
                    allele2_grad_hess(n, x0, x1, eps, g0, g1, h00, h01, h11);
                },
                iterations, maf, p, q);
}

}  // namespace kg
