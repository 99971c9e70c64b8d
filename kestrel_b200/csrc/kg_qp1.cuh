// kg_qp1.cuh — the simplex QP of the SQP step (src/sqp.rs:112-250) solved by
// one thread: min 1/2 y'Qy + c'y subject to y >= 0, sum y = 1, from y0, by the
// reference's active-set method.  Each iteration factors the free block of Q
// with the GMW81-modified LDL^T (src/cholesky.rs:6-65), solves it for the
// gradient and for the ones vector, and either releases the variable with the
// most negative multiplier or steps to the first blocking bound.
//
// It computes what the row-parallel form (qp_simplex_rows in kg_rowsolve.cuh)
// computes, operation for operation and in the same order (the same FMAs,
// divisions and sequential sums), so both give the same bits; with a thread
// per slot a warp serves 32 pairs' QPs instead of two.  Q is read where it
// lies (the slot's QP buffer, through L1); L and the vectors are fixed-size
// arrays indexed by loop counters that unroll, so they stay in registers or
// the thread's local memory.
#pragma once

#include "kg_solver.cuh"

namespace kg {

// GMW81-modified LDL^T of the free block (mask F, nf free) of the 9 x 9 Q,
// which it reads inside that block only; L unit lower triangular with
// identity rows and columns for the fixed variables, d their diagonal 1.
__device__ __forceinline__ void ldl_gmw_thread(const double (*Q)[9], unsigned F, int nf, double (&L)[9][9],
                                               double (&d)[9]) {
    double gamma = 0.0, xi = 0.0;
#pragma unroll
    for (int r = 0; r < 9; r++) {
        if (!((F >> r) & 1u)) continue;
        double diag = fabs(Q[r][r]);
        if (!(diag >= 0.0)) diag = 0.0;
        gamma = fmax(gamma, diag);
        double off = 0.0;
#pragma unroll
        for (int j = r + 1; j < 9; j++)
            if ((F >> j) & 1u) off = fmax(off, fabs(Q[r][j]));
        if (!(off >= 0.0)) off = 0.0;
        xi = fmax(xi, off);
    }
    const double eps = 2.220446049250313e-16;
    const double delta = eps * fmax(1.0, gamma + xi);
    const double t = sqrt((double)nf * (double)nf - 1.0);
    const double ratio = (nf <= 1) ? 0.0 : xi / t;
    const double beta2 = fmax(fmax(gamma, ratio), eps);
#pragma unroll
    for (int i = 0; i < 9; i++) {
        d[i] = 0.0;
#pragma unroll
        for (int j = 0; j < 9; j++) L[i][j] = 0.0;
    }
#pragma unroll
    for (int j = 0; j < 9; j++) {
        if (!((F >> j) & 1u)) {
            d[j] = 1.0;
            L[j][j] = 1.0;
            continue;
        }
        double p[9];
        double sjj = 0.0;
#pragma unroll
        for (int s = 0; s < j; s++) {
            p[s] = d[s] * L[j][s];
            sjj = fma(p[s], L[j][s], sjj);
        }
        const double cjj = Q[j][j] - sjj;
        double c[9];
        double theta = 0.0;
#pragma unroll
        for (int i = j + 1; i < 9; i++) {
            if (!((F >> i) & 1u)) continue;
            double sij = 0.0;
#pragma unroll
            for (int s = 0; s < j; s++) sij = fma(p[s], L[i][s], sij);
            c[i] = Q[i][j] - sij;
            double a = fabs(c[i]);
            if (!(a >= 0.0)) a = 0.0;
            theta = fmax(theta, a);
        }
        const double dj = fmax(fmax(fabs(cjj), theta * theta / beta2), delta);
#pragma unroll
        for (int i = j + 1; i < 9; i++)
            if ((F >> i) & 1u) L[i][j] = c[i] / dj;
        L[j][j] = 1.0;
        d[j] = dj;
    }
}

// L D L^T z = b for two right-hand sides, in the order of ldl_solve2_rows.
__device__ __forceinline__ void ldl_solve2_thread(const double (&L)[9][9], const double (&d)[9], double (&b0)[9],
                                                  double (&b1)[9]) {
    double f0[9], f1[9];
#pragma unroll
    for (int i = 0; i < 9; i++) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int j = 0; j < i; j++) {
            s0 = fma(f0[j], L[i][j], s0);
            s1 = fma(f1[j], L[i][j], s1);
        }
        f0[i] = b0[i] - s0;
        f1[i] = b1[i] - s1;
    }
#pragma unroll
    for (int i = 0; i < 9; i++) {
        f0[i] = f0[i] / d[i];
        f1[i] = f1[i] / d[i];
    }
#pragma unroll
    for (int i = 8; i >= 0; i--) {
        double t0 = 0.0, t1 = 0.0;
#pragma unroll
        for (int j = i + 1; j < 9; j++) {
            t0 = fma(b0[j], L[j][i], t0);
            t1 = fma(b1[j], L[j][i], t1);
        }
        b0[i] = f0[i] - t0;
        b1[i] = f1[i] - t1;
    }
}

// The QP from y0 (y0 and y may alias).  Returns the iteration count.
__device__ inline int qp_simplex_thread(const double (*Q)[9], const double (&c)[9], const double* y0,
                                        const Tune& tu, double* y) {
    unsigned work = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        y[i] = y0[i];
        if (y[i] == 0.0) work |= 1u << i;
    }
    for (int it = 0; it < tu.qp_max_iter; it++) {
        normalise9(y);
        const unsigned F = (~work) & 0x1FFu;
        const int nf = __popc(F);
        if (nf == 0) return it;
        // the free block's gradient c_f + Q_f y_f and the ones vector (the
        // factorisation below reads Q inside the free block only)
        double gf[9], on[9];
#pragma unroll
        for (int r = 0; r < 9; r++) {
            const bool rf = (F >> r) & 1u;
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 9; j++)
                if (rf && ((F >> j) & 1u)) s = fma(Q[r][j], y[j], s);
            gf[r] = rf ? c[r] + s : 0.0;
            on[r] = rf ? 1.0 : 0.0;
        }
        double L[9][9], d[9];
        ldl_gmw_thread(Q, F, nf, L, d);
        ldl_solve2_thread(L, d, gf, on);
        double sg = 0.0, so = 0.0;
#pragma unroll
        for (int i = 0; i < 9; i++)
            if ((F >> i) & 1u) { sg += gf[i]; so += on[i]; }
        const double lambda = sg / so;
        double g2[9];
        double m = 0.0;
        bool m_nan = false;
#pragma unroll
        for (int i = 0; i < 9; i++) {
            g2[i] = lambda * on[i] - gf[i];
            const double a = fabs(g2[i]);
            if (isnan(a)) m_nan = true;
            else m = fmax(m, a);
        }
        if (!m_nan && m <= tu.qp_zero_search_tol) {
            if (nf == 9) return it;
            // the full gradient c + Q y
            double gq[9];
#pragma unroll
            for (int r = 0; r < 9; r++) gq[r] = c[r] + dot_fma(9, Q[r], y);
            int best = -1;
            double gb = 0.0;
#pragma unroll
            for (int i = 0; i < 9; i++)
                if (((work >> i) & 1u) && (best < 0 || gq[i] < gb)) { best = i; gb = gq[i]; }
            if (gb - lambda >= -tu.qp_conv_tol) return it;
            work &= ~(1u << best);
        } else {
            double pv[9];
#pragma unroll
            for (int i = 0; i < 9; i++) pv[i] = ((work >> i) & 1u) ? 0.0 : g2[i];
            double alpha = 1.0;
            int block = -1;
#pragma unroll
            for (int i = 0; i < 9; i++) {
                if (pv[i] < 0.0) {
                    const double a = -y[i] / pv[i];
                    if (a < alpha) { alpha = a; block = i; }
                }
            }
#pragma unroll
            for (int i = 0; i < 9; i++) y[i] = fmax(y[i] + alpha * pv[i], 0.0);
            if (block >= 0) {
                work |= 1u << block;
#pragma unroll
                for (int i = 0; i < 9; i++)
                    if (i == block) y[i] = 0.0;
            }
        }
    }
    return tu.qp_max_iter;
}

}  // namespace kg
