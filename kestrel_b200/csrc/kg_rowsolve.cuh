// kg_rowsolve.cuh — the 9x9 FP64 simplex QP run row-parallel by one warp.
//
// Lane r (r < 9) owns row r of the 9x9 matrices (Hessian, LDL^T factor) in
// registers; 9-vectors are warp-uniform register arrays.  Instead of
// compacting the free variables as the reference does (src/sqp.rs:134-159),
// the working-set rows and columns are masked to zero: the masked entries
// contribute exact zeros to every fma chain and maximum, so the free block is
// factored and solved with the same operations in the same order as the
// reference's compacted form (modify_gmw_n src/cholesky.rs:6-65,
// solve_ldl_mut_n :105-140, solve_qp_active_set src/sqp.rs:112-250).
#pragma once

#include <cstdint>
#include <cmath>

#include "kg_solver.cuh"

namespace kg {

constexpr unsigned FULL_MASK = 0xffffffffu;

// The lanes that run one pair's solver: a whole warp (W = 32) or a half-warp
// (W = 16, two pairs per warp).  Row r of the 9x9 matrices lives in the
// group's lane r; 9-vectors are uniform across the group.
template <int W>
struct Grp {
    unsigned mask;
    __device__ __forceinline__ double bcast(double v, int src) const { return __shfl_sync(mask, v, src, W); }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
};
using WarpGrp = Grp<32>;
using HalfGrp = Grp<16>;

__device__ __forceinline__ double bcast(double v, int src) { return __shfl_sync(FULL_MASK, v, src); }

// Group-uniform copy of the values held by lanes 0..8.
template <class G>
__device__ __forceinline__ void gather9(const G& g, double v, double* out) {
#pragma unroll
    for (int i = 0; i < 9; i++) out[i] = g.bcast(v, i);
}
__device__ __forceinline__ void gather9(double v, double* out) { gather9(WarpGrp{FULL_MASK}, v, out); }

// Element `r` (a lane index) of a uniform register vector.
__device__ __forceinline__ double pick9(const double* v, int r) {
    double o = 0.0;
#pragma unroll
    for (int i = 0; i < 9; i++)
        if (i == r) o = v[i];
    return o;
}


// Maximum over the group's lanes of non-negative values (NaN counts as 0, as
// fmax drops it): for doubles >= 0 the bit patterns order as the values, so
// two 32-bit reductions (high words, then the low words of the lanes holding
// the largest high word) give the maximum without a shuffle tree.
template <class G>
__device__ __forceinline__ double group_max_nonneg(const G& g, double v) {
    if (!(v >= 0.0)) v = 0.0;
    const unsigned hi = (unsigned)__double2hiint(v), lo = (unsigned)__double2loint(v);
    const unsigned mh = __reduce_max_sync(g.mask, hi);
    const unsigned ml = __reduce_max_sync(g.mask, hi == mh ? lo : 0u);
    return __hiloint2double((int)mh, (int)ml);
}

// GMW81-modified LDL^T of the masked matrix: q = this lane's row of Q with
// free mask F (nf free variables).  Returns this lane's row of L and the
// uniform diagonal d.
template <class G>
__device__ __forceinline__ void ldl_gmw_rows(const G& g, const double* q, unsigned F, int nf, int r,
                                             double* Lr, double* d) {
    const bool rf = (r < 9) && ((F >> r) & 1u);
    double diag = 0.0, off = 0.0;
#pragma unroll
    for (int j = 0; j < 9; j++) {
        const bool jf = (F >> j) & 1u;
        if (rf && j == r) diag = fabs(q[j]);
        if (rf && jf && j > r) off = fmax(off, fabs(q[j]));
    }
    const double gamma = group_max_nonneg(g, diag);
    const double xi = group_max_nonneg(g, off);
    const double eps = 2.220446049250313e-16;
    const double delta = eps * fmax(1.0, gamma + xi);
    const double t = sqrt((double)nf * (double)nf - 1.0);
    const double ratio = (nf <= 1) ? 0.0 : xi / t;
    const double beta2 = fmax(fmax(gamma, ratio), eps);
    double p[9];
#pragma unroll
    for (int j = 0; j < 9; j++) { Lr[j] = 0.0; d[j] = 0.0; p[j] = 0.0; }
#pragma unroll
    for (int j = 0; j < 9; j++) {
        if (!((F >> j) & 1u)) {
            d[j] = 1.0;
            if (r == j) Lr[j] = 1.0;
            continue;
        }
        double sjj = 0.0;
#pragma unroll
        for (int s = 0; s < j; s++) {
            const double ljs = g.bcast(Lr[s], j);
            p[s] = d[s] * ljs;
            sjj = fma(p[s], ljs, sjj);
        }
        const double cjj = g.bcast(q[j], j) - sjj;
        double sij = 0.0;
#pragma unroll
        for (int s = 0; s < j; s++) sij = fma(p[s], Lr[s], sij);
        const double cij = q[j] - sij;
        const bool act = rf && (r > j);
        const double theta = group_max_nonneg(g, act ? fabs(cij) : 0.0);
        const double dj = fmax(fmax(fabs(cjj), theta * theta / beta2), delta);
        if (act) Lr[j] = cij / dj;
        if (r == j) Lr[j] = 1.0;
        d[j] = dj;
    }
}

// Solves L D L^T z = b for two right-hand sides held one element per lane
// (b0, b1 for this lane's row), in the reference's summation order.
template <class G>
__device__ __forceinline__ void ldl_solve2_rows(const G& g, const double* Lr, const double* d, int r, double& b0,
                                                double& b1) {
    // forward: b_i -= sum_{j<i} b_j L[i][j]
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int j = 0; j < 9; j++) {
        const double f0 = g.bcast(b0 - s0, j);
        const double f1 = g.bcast(b1 - s1, j);
        if (r > j) {
            s0 = fma(f0, Lr[j], s0);
            s1 = fma(f1, Lr[j], s1);
        }
    }
    b0 -= s0;
    b1 -= s1;
    const double dr = pick9(d, r);
    b0 /= dr;
    b1 /= dr;
    // backward: b_i -= sum_{j>i} b_j L[j][i], j ascending
    double fin0[9], fin1[9];
#pragma unroll
    for (int i = 8; i >= 0; i--) {
        double t0 = 0.0, t1 = 0.0;
#pragma unroll
        for (int j = i + 1; j < 9; j++) {
            const double lji = g.bcast(Lr[i], j);
            t0 = fma(fin0[j], lji, t0);
            t1 = fma(fin1[j], lji, t1);
        }
        fin0[i] = g.bcast(b0, i) - t0;
        fin1[i] = g.bcast(b1, i) - t1;
    }
    b0 = pick9(fin0, r);
    b1 = pick9(fin1, r);
}

// min 1/2 y'Qy + c'y s.t. y >= 0, sum y = 1, from y0.  Hr: this lane's row of Q;
// lane: the lane's index within the group.  Returns the iteration count the
// reference returns beside y (src/sqp.rs:112-250).
template <class G>
__device__ inline int qp_simplex_rows(const G& grp, const double* Hr, const double* c, const double* y0,
                                      const Tune& tu, int lane, double* y) {
    unsigned work = 0;
#pragma unroll
    for (int i = 0; i < 9; i++) {
        y[i] = y0[i];
        if (y[i] == 0.0) work |= 1u << i;
    }
    const int r = lane;
    for (int it = 0; it < tu.qp_max_iter; it++) {
        normalise9(y);
        const unsigned F = (~work) & 0x1FFu;
        const int nf = __popc(F);
        if (nf == 0) return it;
        const bool rf = (r < 9) && ((F >> r) & 1u);
        double q[9];
#pragma unroll
        for (int j = 0; j < 9; j++) q[j] = (rf && ((F >> j) & 1u)) ? Hr[j] : 0.0;
        // g_f = c_f + Q_f y_f
        double gf = 0.0;
        if (rf) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < 9; j++)
                if ((F >> j) & 1u) s = fma(q[j], y[j], s);
            gf = pick9(c, r) + s;
        }
        double Lr[9], d[9];
        ldl_gmw_rows(grp, q, F, nf, r, Lr, d);
        double ones = rf ? 1.0 : 0.0;
        ldl_solve2_rows(grp, Lr, d, r, gf, ones);
        double gfu[9], onu[9];
        gather9(grp, gf, gfu);
        gather9(grp, ones, onu);
        double sg = 0.0, so = 0.0;
#pragma unroll
        for (int i = 0; i < 9; i++)
            if ((F >> i) & 1u) { sg += gfu[i]; so += onu[i]; }
        const double lambda = sg / so;
        double g2[9];
        double m = 0.0;
        bool m_nan = false;
#pragma unroll
        for (int i = 0; i < 9; i++) {
            g2[i] = lambda * onu[i] - gfu[i];
            const double a = fabs(g2[i]);
            if (isnan(a)) m_nan = true;
            else m = fmax(m, a);
        }
        if (!m_nan && m <= tu.qp_zero_search_tol) {
            if (nf == 9) return it;
            // full gradient c + Q y
            double gq = 0.0;
            if (r < 9) gq = pick9(c, r) + dot_fma(9, Hr, y);
            double gqu[9];
            gather9(grp, gq, gqu);
            int best = -1;
#pragma unroll
            for (int i = 0; i < 9; i++)
                if (((work >> i) & 1u) && (best < 0 || gqu[i] < pick9(gqu, best))) best = i;
            if (pick9(gqu, best) - lambda >= -tu.qp_conv_tol) return it;
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
