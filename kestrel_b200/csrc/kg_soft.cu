// kg_soft.cu — the GL/PL estimator on soft genotype likelihoods
// (src/wrapper.rs:89-330 with src/mixture.rs:9-140 and src/coefficients.rs:
// 40-141): per-site allele frequencies by the HWE SQP on the samples'
// likelihoods, then for every pair the Jacquard SQP on the rows L_s = sum over
// (gx, gy) of GLx(gx) GLy(gy) m(gx, gy) of its sites.
//
// Layout: biallelic likelihoods double [sample][site][3] (0/0, 0/1, 1/1;
// linear scale; a NaN marks a missing sample) as loaded; the kept sites'
// likelihoods are also packed as FP32 [sample][kept site] float4 records
// (the three likelihoods and a zero; all three NaN when missing), beside the
// kept sites' FP32 (REF, ALT) frequency pairs.  Tri- and tetra-allelic sites: double [sample][site][6] and
// [sample][site][10] in the VCF genotype order.
//
// A warp per pair, lanes over the kept sites; the SQP itself is FP64.  Its
// evaluations (f, g and H at a point) of the biallelic sites run in one of two
// forms:
//   * FP32 (the default, KG_PREC_FP32C): from the FP32 likelihoods, which stay
//     L2-resident for cohorts of a few hundred samples, each site's row L is
//     formed from the pair's nine likelihood products in closed form; d =
//     eps + L.x with the FP32 hi parts of x, the sums in FP32 promoted to FP64
//     (gradient and objective every 8 sites, Hessian every 32 into the lane's
//     shared memory), and the lo parts of x restored to first order in FP64;
//     near convergence the objective change is summed as log(d / d_old), as
//     on the hard-call path.  A pair whose FP32 condition estimate exceeds
//     COND_RECHECK, or whose KKT residual stalls below 1e-6 three times, is
//     re-evaluated in FP64 and stays FP64 (the hard-call path's rule).
//   * FP64 (KG_PREC_FP64, and escalated pairs): from the FP64 likelihoods,
//     each row the sum over the nine genotype pairs of GLx GLy m(gx, gy).
// Tri- and tetra-allelic sites keep the genotypes of the alleles left after
// the frequency cut (src/wrapper.rs:349-409); their rows (G' x G' x 9 terms
// each) are built once per pair in FP64 into the warp's scratch, as the
// reference builds its pair buffer once, and every evaluation adds their FP64
// sums to the biallelic ones.  The shared-memory sums of a warp are 45 rows of
// 33 doubles: the 32 lanes' partials and the warp's total.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <string>
#include <vector>

#include "kestrel_gpu.h"
#include "kg_allele.cuh"
#include "kg_alleleN.cuh"
#include "kg_bulk.cuh"
#include "kg_engine.h"
#include "kg_pair.cuh"
#include "kg_rowsolve.cuh"
#include "kg_solver.cuh"

namespace kg {

#define KG_SOFT_TRY(expr)                                                       \
    do {                                                                        \
        cudaError_t e_ = (expr);                                                \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);           \
            return e_ == cudaErrorMemoryAllocation ? KG_ENOMEM : KG_ECUDA;      \
        }                                                                       \
    } while (0)

// Thread per site: frequencies (REF, ALT) and the keep flag (both non-zero
// after the maf cut).  Adjacent threads read adjacent sites of a sample.
__device__ __forceinline__ double warp_allsum(double v) {
    // butterfly: every lane adds the same two partials at every level, so all
    // lanes end with the same bits
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// Warp per site: the HWE SQP of the site's frequencies with the samples over
// the lanes (the sums of src/mixture.rs's objective and derivatives reduced
// across the warp; every lane then runs the same solver steps on the same
// values).
__global__ void soft_freq_kernel(const double* __restrict__ gl, int64_t n_samples, int64_t n_sites, double maf,
                                 uint64_t iterations, double* __restrict__ pf, double* __restrict__ qf,
                                 uint8_t* __restrict__ keep) {
    const int lane = threadIdx.x & 31;
    const int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (v >= n_sites) return;
    const double eps = make_tune(iterations).epsilon;
    auto rowp = [&](int64_t s) { return gl + (s * n_sites + v) * 3; };
    double called = 0.0;
    for (int64_t s = lane; s < n_samples; s += 32) {
        const double* r = rowp(s);
        called += !(isnan(r[0]) || isnan(r[1]) || isnan(r[2]));
    }
    called = warp_allsum(called);
    double p = 0.0, q = 0.0;
    if (called > 0.0) {
        auto obj = [&](double x0, double x1) {
            double acc = 0.0;
            const double w0 = x0 * x0, w1 = 2.0 * x0 * x1, w2 = x1 * x1;
            for (int64_t s = lane; s < n_samples; s += 32) {
                const double* r = rowp(s);
                const double l0 = r[0], l1 = r[1], l2 = r[2];
                if (isnan(l0) || isnan(l1) || isnan(l2)) continue;
                acc += log(fma(w2, l2, fma(w1, l1, fma(w0, l0, eps))));
            }
            return -warp_allsum(acc) / called;
        };
        auto gh = [&](double x0, double x1, double& g0, double& g1, double& h00, double& h01, double& h11) {
            double zg0 = 0.0, zg1 = 0.0, z00 = 0.0, z01 = 0.0, z11 = 0.0;
            for (int64_t s = lane; s < n_samples; s += 32) {
                const double* r = rowp(s);
                const double l0 = r[0], l1 = r[1], l2 = r[2];
                if (isnan(l0) || isnan(l1) || isnan(l2)) continue;
                const double lx0 = fma(l1, x1, fma(l0, x0, 0.0));
                const double lx1 = fma(l2, x1, fma(l1, x0, 0.0));
                const double d = fma(x1, lx1, fma(x0, lx0, eps));
                const double inv = 1.0 / d;
                const double a0 = lx0 * inv, a1 = lx1 * inv;
                zg0 += a0;
                zg1 += a1;
                z00 += 2.0 * a0 * a0 - l0 * inv;
                z01 += 2.0 * a0 * a1 - l1 * inv;
                z11 += 2.0 * a1 * a1 - l2 * inv;
            }
            g0 = -2.0 * warp_allsum(zg0) / called;
            g1 = -2.0 * warp_allsum(zg1) / called;
            h00 = 2.0 * warp_allsum(z00) / called;
            h01 = 2.0 * warp_allsum(z01) / called;
            h11 = 2.0 * warp_allsum(z11) / called;
        };
        allele2_fit(obj, gh, iterations, maf, p, q);
    }
    if (lane == 0) {
        pf[v] = p;
        qf[v] = q;
        keep[v] = (p > 0.0 && q > 0.0) ? 1 : 0;
    }
}

constexpr int SOFT_WARPS = 4;
constexpr int HS = 33;   // shared-memory stride of the Hessian sums: 32 lane partials, then the warp total
// A warp's shared memory: the Hessian sums (45 rows of HS doubles, padded to
// 16 bytes), then per lane SOFT_STAGES slots of 48 bytes for the FP32 form's
// prefetched site (the two samples' float4 records and the (p, q) pair).
constexpr int SOFT_STAGES = 3;
constexpr int SOFT_SUMS_BYTES = (45 * HS * 8 + 15) / 16 * 16;
constexpr int SOFT_WARP_SMEM = SOFT_SUMS_BYTES + 32 * SOFT_STAGES * 48;
constexpr int SOFT_SMEM = SOFT_WARPS * SOFT_WARP_SMEM;

// ---------------------------------------------------------- tri / tetra
// A loaded tri- or tetra-allelic site after its frequency fit: G' genotypes of
// the remaining alleles (0: discarded), the original genotype index of each,
// and the site's G' x G' rows m[g'x][g'y] (stride ML_SOFT_ROWS rows).
constexpr int SOFT_MULTI_ROWS = 100;

struct SoftMultiDev {
    const double* gl[2];      // [sample][site][G0] of the tri- and of the tetra-allelic sites
    int64_t n[2];             // their site counts
    int64_t total;            // n[0] + n[1]: tri-allelic sites first
    const int32_t* gk;        // per site: G' (0 = discarded)
    const uint8_t* gidx;      // per site: [10] original genotype of reduced genotype g'
    const double* rows;       // per site: SOFT_MULTI_ROWS x 9
    double* scratch;          // per warp: total x 9, the current pair's rows (NaN first entry: no row)
};

// Per-sample likelihood rows of one multi-allelic site (a row with a NaN is a
// missing sample), weight 1: the row source of allele_fit.
struct SoftRows {
    const double* gl;
    int64_t n_samples, n_sites, v;
    int a, g0;
    __device__ int alleles() const { return a; }
    __device__ int rows() const { return (int)n_samples; }
    __device__ double weight(int) const { return 1.0; }
    __device__ bool row(int k, double* l) const {
        const double* r = gl + ((int64_t)k * n_sites + v) * g0;
        bool ok = true;
        for (int g = 0; g < MAXG; g++) {
            l[g] = g < g0 ? r[g] : 0.0;
            ok = ok && !(g < g0 && isnan(l[g]));
        }
        return ok;
    }
};

// Thread per tri-/tetra-allelic site: the frequency fit on the samples'
// likelihoods with the maf cut, the alleles left (in order), each reduced
// genotype's original index and the site's rows; used[0..2] counts the sites
// left with 2, 3, 4 alleles.
__global__ void soft_multi_site_kernel(SoftMultiDev M, int64_t n_samples, double maf, uint64_t iterations,
                                       int32_t* __restrict__ gk, uint8_t* __restrict__ gidx,
                                       double* __restrict__ rows, unsigned long long* __restrict__ used) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M.total) return;
    const int c = t < M.n[0] ? 0 : 1;
    const int64_t v = c == 0 ? t : t - M.n[0];
    SoftRows src;
    src.gl = M.gl[c];
    src.n_samples = n_samples;
    src.n_sites = M.n[c];
    src.v = v;
    src.a = c == 0 ? 3 : 4;
    src.g0 = c == 0 ? 6 : 10;
    double f[MAXA];
    allele_fit(src, iterations, maf, f);
    int keep[MAXA], na = 0;
    double fk[MAXA] = {0.0, 0.0, 0.0, 0.0};
    for (int a = 0; a < src.a; a++)
        if (f[a] > 0.0) {
            keep[na] = a;
            fk[na] = f[a];
            na++;
        }
    if (na < 2) {
        gk[t] = 0;
        return;
    }
    const int g = na * (na + 1) / 2;
    gk[t] = g;
    int k = 0;
    for (int j = 0; j < na; j++)
        for (int i = 0; i <= j; i++) gidx[MAXG * t + k++] = (uint8_t)(keep[j] * (keep[j] + 1) / 2 + keep[i]);
    double* R = rows + (int64_t)SOFT_MULTI_ROWS * 9 * t;
    for (int gx = 0; gx < g; gx++) {
        int i, j;
        genotype_alleles(gx, i, j);
        for (int gy = 0; gy < g; gy++) {
            int a, b;
            genotype_alleles(gy, a, b);
            iis_row(i, j, a, b, fk[0], fk[1], fk[2], fk[3], R + 9 * (gx * g + gy));
        }
    }
    atomicAdd(&used[na - 2], 1ull);
}

// The pair's rows at the multi-allelic sites, in FP64, into the warp's
// scratch: sum over the remaining genotypes of GLx(gx) GLy(gy) m[gx][gy]
// (gx outer, gy inner, as src/mixture.rs:9-60 accumulates); NaN first entry
// when a sample is missing or the site was discarded.  Returns the warp's count
// of rows.
__device__ __noinline__ int64_t soft_multi_build(const SoftMultiDev M, int64_t x, int64_t y, int lane, double* R) {
    int64_t m = 0;
    for (int64_t t = lane; t < M.total; t += 32) {
        double* o = R + 9 * t;
        const int g = M.gk[t];
        bool ok = g > 0;
        double L[9];
#pragma unroll
        for (int k = 0; k < 9; k++) L[k] = 0.0;
        if (ok) {
            const int c = t < M.n[0] ? 0 : 1;
            const int64_t v = c == 0 ? t : t - M.n[0];
            const int g0 = c == 0 ? 6 : 10;
            const double* lx = M.gl[c] + (x * M.n[c] + v) * g0;
            const double* ly = M.gl[c] + (y * M.n[c] + v) * g0;
            const uint8_t* gi = M.gidx + MAXG * t;
            const double* mm = M.rows + (int64_t)SOFT_MULTI_ROWS * 9 * t;
            for (int gx = 0; gx < g && ok; gx++) {
                const double ax = lx[gi[gx]];
                for (int gy = 0; gy < g; gy++) {
                    const double gg = ax * ly[gi[gy]];
#pragma unroll
                    for (int k = 0; k < 9; k++) L[k] = fma(gg, mm[9 * (gx * g + gy) + k], L[k]);
                }
            }
#pragma unroll
            for (int k = 0; k < 9; k++) ok = ok && !isnan(L[k]);
        }
        if (ok) {
#pragma unroll
            for (int k = 0; k < 9; k++) o[k] = L[k];
            m++;
        } else {
            o[0] = CUDART_NAN;
        }
    }
    for (int off = 16; off > 0; off >>= 1) m += __shfl_xor_sync(0xffffffffu, m, off);
    __syncwarp();   // the rows are read by every lane's evaluations
    return m;
}

// Adds the pair's multi-allelic rows at xt to the warp's totals, in FP64:
// G (warp-uniform), the 45 Hessian totals at hs[a * HS + 32], F (sum log d, or
// sum log(d / d_old) with d_old at xc in a difference pass) and n.
__device__ __noinline__ void soft_multi_add(const double* R, int64_t total, const double* xt, const double* xc,
                                            bool diff, double eps, int lane, double* hs, double* G, double& F,
                                            int64_t& n) {
    double g[9], f = 0.0;
#pragma unroll
    for (int i = 0; i < 9; i++) g[i] = 0.0;
    int64_t m = 0;
    for (int a = 0; a < 45; a++) hs[a * HS + lane] = 0.0;
    for (int64_t t = lane; t < total; t += 32) {
        const double* L = R + 9 * t;
        if (isnan(L[0])) continue;
        double d = eps;
#pragma unroll
        for (int i = 0; i < 9; i++) d = fma(xt[i], L[i], d);
        const double r = 1.0 / d;
        double b[9];
#pragma unroll
        for (int i = 0; i < 9; i++) {
            g[i] = fma(L[i], r, g[i]);
            b[i] = L[i] * r;
        }
        int a = 0;
#pragma unroll
        for (int i = 0; i < 9; i++)
#pragma unroll
            for (int j = i; j < 9; j++, a++) hs[a * HS + lane] = fma(b[i], b[j], hs[a * HS + lane]);
        if (!diff) {
            f += log(d);
        } else {
            double dc = eps, dl = 0.0;
#pragma unroll
            for (int i = 0; i < 9; i++) {
                dc = fma(xc[i], L[i], dc);
                dl = fma(xt[i] - xc[i], L[i], dl);
            }
            f += log1p(dl / dc);
        }
        m++;
    }
    for (int off = 16; off > 0; off >>= 1) {
        f += __shfl_xor_sync(0xffffffffu, f, off);
        m += __shfl_xor_sync(0xffffffffu, m, off);
#pragma unroll
        for (int i = 0; i < 9; i++) g[i] += __shfl_xor_sync(0xffffffffu, g[i], off);
    }
    __syncwarp();
    for (int a = 0; a < 45; a++) {
        double h = hs[a * HS + lane];
        for (int off = 16; off > 0; off >>= 1) h += __shfl_xor_sync(0xffffffffu, h, off);
        if (lane == 0) hs[a * HS + 32] += h;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 9; i++) G[i] += g[i];
    F += f;
    n += m;
}

// The Hessian total (i, j) of the upper triangle, row-major.
__device__ __forceinline__ double htotal(const double* hs, int i, int j) {
    const int i0 = i < j ? i : j, j0 = i < j ? j : i;
    return hs[(i0 * 9 - i0 * (i0 - 1) / 2 + (j0 - i0)) * HS + 32];
}

// The warp's 45 Hessian totals from the lanes' partials: hs[a * HS + 32].
__device__ __forceinline__ void hessian_totals(double* hs, int lane) {
    __syncwarp();
    for (int a = 0; a < 45; a++) {
        double h = hs[a * HS + lane];
        for (int off = 16; off > 0; off >>= 1) h += __shfl_xor_sync(0xffffffffu, h, off);
        if (lane == 0) hs[a * HS + 32] = h;
    }
    __syncwarp();
}

// f, g and this lane's Hessian row at x over the pair's rows (-(1/n) sum log(eps
// + L.x), -(1/n) sum L r, (1/n) sum L L' r^2, r = 1/(eps + L.x)); n = rows
// without a NaN.  hs: the warp's Hessian sums in shared memory; R, nm: the
// pair's multi-allelic rows.
__device__ __noinline__ int64_t soft_evaluate(const double* __restrict__ gl, int64_t n_sites,
                                              const int32_t* __restrict__ kept, const double* __restrict__ kp,
                                              const double* __restrict__ kq, int64_t nk, int64_t x, int64_t y,
                                              const double* xv, double eps, int lane, double* hs, const double* R,
                                              int64_t nm, PairEval& ev) {
    double f = 0.0, g[9];
#pragma unroll
    for (int i = 0; i < 9; i++) g[i] = 0.0;
    for (int a = 0; a < 45; a++) hs[a * HS + lane] = 0.0;
    int64_t n = 0;
    for (int64_t k = lane; k < nk; k += 32) {
        const int64_t v = kept[k];
        const double* lx = gl + (x * n_sites + v) * 3;
        const double* ly = gl + (y * n_sites + v) * 3;
        const double ax[3] = {lx[0], lx[1], lx[2]}, ay[3] = {ly[0], ly[1], ly[2]};
        if (isnan(ax[0] + ax[1] + ax[2] + ay[0] + ay[1] + ay[2])) continue;
        const double p = kp[k], q = kq[k];
        double L[9];
#pragma unroll
        for (int i = 0; i < 9; i++) L[i] = 0.0;
#pragma unroll
        for (int gx = 0; gx < 3; gx++)
#pragma unroll
            for (int gy = 0; gy < 3; gy++) {
                const double w = ax[gx] * ay[gy];
                double m[9];
                cls_row(gx, gy, p, q, m);
#pragma unroll
                for (int i = 0; i < 9; i++) L[i] = fma(w, m[i], L[i]);
            }
        double d = eps;
#pragma unroll
        for (int i = 0; i < 9; i++) d = fma(xv[i], L[i], d);
        f += log(d);
        const double r = 1.0 / d;
        double b[9];
#pragma unroll
        for (int i = 0; i < 9; i++) {
            g[i] = fma(L[i], r, g[i]);
            b[i] = L[i] * r;
        }
        int a = 0;
#pragma unroll
        for (int i = 0; i < 9; i++)
#pragma unroll
            for (int j = i; j < 9; j++, a++) hs[a * HS + lane] = fma(b[i], b[j], hs[a * HS + lane]);
        n++;
    }
    // warp sums (fixed butterfly order)
    for (int off = 16; off > 0; off >>= 1) {
        f += __shfl_xor_sync(0xffffffffu, f, off);
        n += __shfl_xor_sync(0xffffffffu, n, off);
#pragma unroll
        for (int i = 0; i < 9; i++) g[i] += __shfl_xor_sync(0xffffffffu, g[i], off);
    }
    hessian_totals(hs, lane);
    if (nm > 0) soft_multi_add(R, nm, xv, xv, false, eps, lane, hs, g, f, n);
    const double dn = (double)n;
    ev.f = -f / dn;
#pragma unroll
    for (int i = 0; i < 9; i++) ev.g[i] = -g[i] / dn;
    // lane i < 9 takes row i of H
#pragma unroll
    for (int j = 0; j < 9; j++) ev.Hr[j] = lane < 9 ? htotal(hs, lane, j) / dn : 0.0;
    __syncwarp();
    return n;
}

// Packs the kept sites' likelihoods as FP32 [sample][kept][3], all three NaN
// for a missing sample, and the kept frequencies as FP32.
__global__ void soft_pack32_kernel(const double* __restrict__ gl, int64_t n_samples, int64_t n_sites,
                                   const int32_t* __restrict__ kept, const double* __restrict__ kp,
                                   const double* __restrict__ kq, int64_t nk, float4* __restrict__ g32,
                                   float2* __restrict__ pq32) {
    const int64_t total = n_samples * nk;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = t / nk, k = t - s * nk;
        const double* r = gl + (s * n_sites + kept[k]) * 3;
        const bool miss = isnan(r[0]) || isnan(r[1]) || isnan(r[2]);
        g32[t] = miss ? make_float4(CUDART_NAN_F, CUDART_NAN_F, CUDART_NAN_F, 0.f)
                      : make_float4((float)r[0], (float)r[1], (float)r[2], 0.f);
        if (s == 0) pq32[k] = make_float2((float)kp[k], (float)kq[k]);
    }
}

// The FP32 evaluation (see the file comment) at xt; in a difference pass
// (DIFF) the objective is f_old - (1/n) sum log(d / d_old) with d_old at xc.
// hs: the warp's FP64 Hessian sums in shared memory; R, nm: the pair's
// multi-allelic rows, added in FP64 after the lo correction of the biallelic
// sums.  Returns n.  Not inlined: the site loop gets the registers the pair's
// SQP state would hold.
template <bool DIFF>
__device__ __noinline__ int64_t soft_evaluate32(const float4* __restrict__ g32, const float2* __restrict__ pq32,
                                                int64_t nk, int64_t x, int64_t y,
                                                const double* xt, const double* xc, double f_old, double eps,
                                                int lane, double* hs, float4* slots, const double* R, int64_t nm,
                                                PairEval& ev) {
    const bool diff = DIFF;
    float xh[9], sd[9];
#pragma unroll
    for (int i = 0; i < 9; i++) {
        xh[i] = (float)xt[i];
        sd[i] = DIFF ? (float)(xt[i] - xc[i]) : 0.f;
    }
    double G[9], F = 0.0;
    float g[9], h[45], o = 0.f;
#pragma unroll
    for (int i = 0; i < 9; i++) { G[i] = 0.0; g[i] = 0.f; }
#pragma unroll
    for (int a = 0; a < 45; a++) h[a] = 0.f;
    for (int a = 0; a < 45; a++) hs[a * HS + lane] = 0.0;
    const float4* lx = g32 + x * nk;
    const float4* ly = g32 + y * nk;
    const float e32 = (float)eps;
    const int nk32 = (int)nk;
    int64_t n = 0;
    // Warp-uniform iterations (a lane past the end or at a missing sample
    // skips the site), so that the FP64 flushes below run once per warp.  The
    // site two iterations ahead is copied by cp.async into the lane's slots:
    // the prefetch holds no registers.
    float4* my = slots + lane * (3 * SOFT_STAGES);
    const uint32_t my0 = smem_u32(my);
    auto issue = [&](int it2) {
        const int k2 = lane + 32 * it2;
        if (k2 < nk32) {
            const uint32_t d = my0 + 48u * (uint32_t)(it2 % SOFT_STAGES);
            cp_async16(d, lx + k2);
            cp_async16(d + 16u, ly + k2);
            cp_async8(d + 32u, pq32 + k2);
        }
        cp_async_commit();
    };
    const int iters = (nk32 + 31) >> 5;
    issue(0);
    issue(1);
    for (int it = 0; it < iters; it++) {
        issue(it + 2);
        cp_async_wait<2>();   // this iteration's site has landed
        const int k = lane + 32 * it;
        const float4* st = my + 3 * (it % SOFT_STAGES);
        float4 X = make_float4(CUDART_NAN_F, 0.f, 0.f, 0.f), Y = X;
        float2 PQ = make_float2(0.f, 0.f);
        if (k < nk32) {
            X = st[0];
            Y = st[1];
            PQ = *reinterpret_cast<const float2*>(st + 2);
        }
        const float X0 = X.x, X1 = X.y, X2 = X.z, Y0 = Y.x, Y1 = Y.y, Y2 = Y.z;
        const float p = PQ.x, q = PQ.y;
        // a missing sample has all three NaN (and so has a lane past the end)
        if (!isnan(X0) && !isnan(Y0)) {
            // L = sum over (gx, gy) of GLx(gx) GLy(gy) m(gx, gy), the nine rows
            // of the biallelic conditional table (cls_row) gathered by entry
            const float A = X0 * Y0, B = X2 * Y2, C = X0 * Y2, D = X2 * Y0, E = X0 * Y1;
            const float Fx = X2 * Y1, Gx = X1 * Y0, Hx = X1 * Y2, I = X1 * Y1;
            const float p2 = p * p, q2 = q * q, pq = p * q;
            const float p2q = p2 * q, pq2 = p * q2;
            const float S2 = fmaf(A, p2, B * q2);
            const float S3 = fmaf(A, p2 * p, B * (q2 * q));
            float L[9];
            L[0] = fmaf(A, p, B * q);
            L[1] = fmaf(C + D, pq, S2);
            L[2] = fmaf(E + Fx, pq, S2);
            L[3] = fmaf(2.0f * E, p2q, fmaf(2.0f * Fx, pq2, fmaf(C, pq2, fmaf(D, p2q, S3))));
            L[4] = fmaf(Gx + Hx, pq, S2);
            L[5] = fmaf(2.0f * Gx, p2q, fmaf(2.0f * Hx, pq2, fmaf(C, p2q, fmaf(D, pq2, S3))));
            L[6] = fmaf(2.0f * I, pq, S2);
            L[7] = fmaf(I, p2q + pq2, fmaf(Fx + Hx, pq2, fmaf(E + Gx, p2q, S3)));
            L[8] = fmaf(4.0f * I, p2 * q2,
                        fmaf(2.0f * (Fx + Hx), pq2 * q,
                             fmaf(2.0f * (E + Gx), p2q * p, fmaf(C + D, p2 * q2, fmaf(A, p2 * p2, B * (q2 * q2))))));
            const float d = dot9_eps(L, xh, e32);
            const float r = rcp_approx(d);
            float b[9];
#pragma unroll
            for (int i = 0; i < 9; i++) {
                b[i] = L[i] * r;
                g[i] += b[i];
            }
            int a = 0;
#pragma unroll
            for (int i = 0; i < 9; i++)
#pragma unroll
                for (int j = i; j < 9; j++, a++) h[a] = fmaf(b[i], b[j], h[a]);
            if (!diff) {
                o += lg2_approx(d);
            } else {
                float dl = 0.f;
#pragma unroll
                for (int i = 0; i < 9; i++) dl = fmaf(L[i], sd[i], dl);
                o += neg_log1m(dl * r);
            }
            n++;
        }
        if ((it & 7) == 7) {
#pragma unroll
            for (int i = 0; i < 9; i++) { G[i] += (double)g[i]; g[i] = 0.f; }
            F += (double)o;
            o = 0.f;
        }
        if ((it & 31) == 31) {
#pragma unroll
            for (int a2 = 0; a2 < 45; a2++) {
                hs[a2 * HS + lane] += (double)h[a2];
                h[a2] = 0.f;
                asm volatile("" ::: "memory");   // one read-modify-write at a time: no register peak
            }
        }
    }
    cp_async_wait<0>();   // no copy outstanding into the slots (they are past the last site)
#pragma unroll
    for (int i = 0; i < 9; i++) G[i] += (double)g[i];
    F += (double)o;
#pragma unroll
    for (int a = 0; a < 45; a++) hs[a * HS + lane] += (double)h[a];
    // warp sums (fixed butterfly order)
    for (int off = 16; off > 0; off >>= 1) {
        F += __shfl_xor_sync(0xffffffffu, F, off);
        n += __shfl_xor_sync(0xffffffffu, n, off);
#pragma unroll
        for (int i = 0; i < 9; i++) G[i] += __shfl_xor_sync(0xffffffffu, G[i], off);
    }
    hessian_totals(hs, lane);
    // the lo parts of x to first order: sum log d gains sum_j lo_j G_j, and
    // G_i loses sum_j H_ij lo_j (a difference pass uses the step's FP32 values)
    double lo[9];
#pragma unroll
    for (int j = 0; j < 9; j++) lo[j] = xt[j] - (double)xh[j];
    double corr = 0.0;
#pragma unroll
    for (int j = 0; j < 9; j++) corr = fma(lo[j], G[j], corr);
    double Gc[9];
#pragma unroll
    for (int i = 0; i < 9; i++) {
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < 9; j++) s = fma(htotal(hs, i, j), lo[j], s);
        Gc[i] = G[i] - s;
    }
    // objective so far in natural-log units (direct: F counted log2 d)
    double fsum = diff ? F : F * 0.69314718055994530942 + corr;
    if (nm > 0) soft_multi_add(R, nm, xt, xc, diff, eps, lane, hs, Gc, fsum, n);
    const double dn = (double)n;
    ev.f = diff ? f_old - fsum / dn : -fsum / dn;
#pragma unroll
    for (int i = 0; i < 9; i++) ev.g[i] = -Gc[i] / dn;
#pragma unroll
    for (int j = 0; j < 9; j++) ev.Hr[j] = lane < 9 ? htotal(hs, lane, j) / dn : 0.0;
    __syncwarp();
    return n;
}

// Warp per output row of the first ns samples (x-major, y >= x), taken from a
// counter; the Jacquard SQP of src/sqp.rs:49-93 in FP64 on FP32 evaluations
// (prec64 = 0) or FP64 ones.  stats: [0] grad-Hessian evaluations, [1] of them
// in FP64, [2] pairs escalated to FP64, [3] pair-sites evaluated (summed over
// evaluations), [4] of them in FP64.
__global__ void __launch_bounds__(SOFT_WARPS * 32, 3) soft_pairs_kernel(
    const double* __restrict__ gl, int64_t n_sites, const int32_t* __restrict__ kept, const double* __restrict__ kp,
    const double* __restrict__ kq, const float4* __restrict__ g32, const float2* __restrict__ pq32, int prec64, int64_t nk, int64_t ns, int64_t n_rows, uint64_t iterations,
    kg_output* out, unsigned long long* next, int* no_rows, unsigned long long* stats, SoftMultiDev M) {
    extern __shared__ __align__(16) unsigned char soft_smem[];   // SOFT_WARP_SMEM per warp
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* hs = reinterpret_cast<double*>(soft_smem + w * SOFT_WARP_SMEM);
    float4* slots = reinterpret_cast<float4*>(soft_smem + w * SOFT_WARP_SMEM + SOFT_SUMS_BYTES);
    // the warp's scratch for its pair's multi-allelic rows
    double* R = M.total > 0 ? M.scratch + ((int64_t)blockIdx.x * SOFT_WARPS + w) * M.total * 9 : nullptr;
    const Tune tu = make_tune(iterations);
    unsigned long long c_gh = 0, c_f64 = 0, c_esc = 0, c_sites = 0, c_sites64 = 0;
    for (;;) {
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(next, 1ull);
        r = __shfl_sync(0xffffffffu, r, 0);
        if ((int64_t)r >= n_rows) break;
        int64_t lo = 0, hi = ns - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (mid * ns - mid * (mid - 1) / 2 <= (int64_t)r) lo = mid;
            else hi = mid - 1;
        }
        const int64_t x = lo, y = x + ((int64_t)r - (x * ns - x * (x - 1) / 2));
        double xv[9];
#pragma unroll
        for (int i = 0; i < 9; i++) xv[i] = x == y ? 0.0 : 1.0 / 9.0;
        if (x == y) { xv[0] = 0.5; xv[6] = 0.5; }
        normalise9(xv);
        bool fp64 = prec64 != 0;
        if (M.total > 0) soft_multi_build(M, x, y, lane, R);
        // one evaluation at xt: FP64, or FP32 (a difference pass relative to xc
        // and the objective f_old there when diff)
        PairEval ev;
        auto eval = [&](const double* xt, const double* xc, bool diff, double f_old) -> int64_t {
            c_gh++;
            int64_t m;
            if (fp64) {
                c_f64++;
                m = soft_evaluate(gl, n_sites, kept, kp, kq, nk, x, y, xt, tu.epsilon, lane, hs, R, M.total, ev);
                c_sites64 += (unsigned long long)m;
            } else {
                m = diff ? soft_evaluate32<true>(g32, pq32, nk, x, y, xt, xc, f_old, tu.epsilon, lane, hs, slots, R,
                                                 M.total, ev)
                         : soft_evaluate32<false>(g32, pq32, nk, x, y, xt, xc, f_old, tu.epsilon, lane, hs, slots, R,
                                                  M.total, ev);
            }
            c_sites += (unsigned long long)m;
            return m;
        };
        const int64_t n = eval(xv, xv, false, 0.0);
        kg_output* o = out + r;
        if (n == 0) {
            if (lane == 0) {
                o->x = (uint64_t)x;
                o->y = (uint64_t)y;
                for (int i = 0; i < 9; i++) o->jacquard[i] = 0.0;
                o->obj = CUDART_NAN;
                o->iters = 0;
                o->cond = CUDART_NAN;
                atomicOr(no_rows, 1);
            }
            continue;
        }
        double f = ev.f, g[9], Hr[9];
#pragma unroll
        for (int i = 0; i < 9; i++) { g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
        uint64_t iters = tu.sqp_max_iter;
        double cond = CUDART_NAN;
        int near_count = 0;
        for (uint64_t it = 0; it < tu.sqp_max_iter; it++) {
            double resid;
            bool conv = kkt_ok(xv, g, tu.sqp_conv_tol, &resid);
            if (!fp64 && (conv || resid < 1e-6)) {
                if (!conv) near_count++;
                const double c32 = conv ? condition_rows(xv, g, Hr, tu.sqp_conv_tol) : 0.0;
                if (conv ? !(c32 <= COND_RECHECK) : (near_count >= 3)) {
                    // FP64 re-evaluation at the same point; the pair stays FP64
                    fp64 = true;
                    c_esc++;
                    eval(xv, xv, false, 0.0);
                    f = ev.f;
#pragma unroll
                    for (int i = 0; i < 9; i++) { g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
                    conv = kkt_ok(xv, g, tu.sqp_conv_tol, &resid);
                } else if (conv) {
                    iters = it;
                    cond = c32;
                    break;
                }
            }
            if (conv) {
                iters = it;
                cond = condition_rows(xv, g, Hr, tu.sqp_conv_tol);
                break;
            }
            double cr = 0.0;
            if (lane < 9) cr = pick9(g, lane) - dot_fma(9, Hr, xv);
            double c[9], yv[9], p[9];
            gather9(cr, c);
            qp_simplex_rows(WarpGrp{FULL_MASK}, Hr, c, xv, tu, lane, yv);
#pragma unroll
            for (int i = 0; i < 9; i++) p[i] = yv[i] - xv[i];
            const double gp = dot_fma(9, g, p);
            const double tt = tu.bls_sufficient_decrease * gp;
            double alpha = 1.0, xn[9];
            for (int bls = 0;;) {
#pragma unroll
                for (int i = 0; i < 9; i++) xn[i] = xv[i] + alpha * p[i];
                normalise9(xn);
                eval(xn, xv, fabs(alpha * gp) < DIFF_BELOW, f);
                const bool accept = ev.f <= f + alpha * tt;
                bls++;
                if (accept || bls == tu.bls_max_iter) break;
                alpha *= tu.bls_step_size_reduce;
            }
#pragma unroll
            for (int i = 0; i < 9; i++) { xv[i] = xn[i]; g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
            f = ev.f;
        }
        if (lane == 0) {
            o->x = (uint64_t)x;
            o->y = (uint64_t)y;
            for (int i = 0; i < 9; i++) o->jacquard[i] = xv[i];
            o->obj = f;
            o->iters = iters;
            o->cond = cond;
        }
    }
    if (lane == 0) {
        atomicAdd(&stats[0], c_gh);
        atomicAdd(&stats[1], c_f64);
        atomicAdd(&stats[2], c_esc);
        atomicAdd(&stats[3], c_sites);
        atomicAdd(&stats[4], c_sites64);
    }
}

int soft_relatedness(SoftWork& w, const DevBuf& gl, int64_t n_samples, int64_t n_sites, int64_t ns,
                     uint64_t iterations, double maf, kg_output* d_out, cudaStream_t st, std::string& err,
                     int64_t* n_kept, int precision,
                     uint64_t* counters, const SoftMultiInput* multi, int64_t* multi_used) {
    if (!(maf >= 0.0)) maf = 1.0 / (2.0 * (double)n_samples);
    DevBuf &pf = w.pf, &qf = w.qf, &keep = w.keep, &idx = w.idx, &kp = w.kp, &kq = w.kq, &ctr = w.ctr;
    DevBuf &g32 = w.g32, &pq32 = w.pq32, &mgk = w.mgk, &mgidx = w.mgidx, &mrows = w.mrows, &mused = w.mused;
    DevBuf& mscratch = w.mscratch;
    KG_SOFT_TRY((cudaError_t)pf.reserve(sizeof(double) * n_sites));
    KG_SOFT_TRY((cudaError_t)qf.reserve(sizeof(double) * n_sites));
    KG_SOFT_TRY((cudaError_t)keep.reserve((size_t)n_sites));
    soft_freq_kernel<<<(unsigned)((n_sites + 3) / 4), 128, 0, st>>>(gl.as<double>(), n_samples, n_sites, maf,
                                                                        iterations, pf.as<double>(), qf.as<double>(),
                                                                        keep.as<uint8_t>());
    KG_SOFT_TRY(cudaGetLastError());
    // the kept sites, compacted on the host (one small copy each way)
    std::vector<double> hp((size_t)n_sites), hq((size_t)n_sites);
    std::vector<uint8_t> hk((size_t)n_sites);
    KG_SOFT_TRY(cudaMemcpyAsync(hp.data(), pf.p, sizeof(double) * n_sites, cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaMemcpyAsync(hq.data(), qf.p, sizeof(double) * n_sites, cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaMemcpyAsync(hk.data(), keep.p, (size_t)n_sites, cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaStreamSynchronize(st));
    std::vector<int32_t> ki;
    std::vector<double> kpv, kqv;
    for (int64_t v = 0; v < n_sites; v++)
        if (hk[(size_t)v]) {
            ki.push_back((int32_t)v);
            kpv.push_back(hp[(size_t)v]);
            kqv.push_back(hq[(size_t)v]);
        }
    const int64_t nk = (int64_t)ki.size();
    if (n_kept) *n_kept = nk;
    // tri- and tetra-allelic sites: frequencies, remaining alleles, rows
    SoftMultiDev M{};
    M.n[0] = multi ? multi->n3 : 0;
    M.n[1] = multi ? multi->n4 : 0;
    M.gl[0] = multi ? multi->gl3 : nullptr;
    M.gl[1] = multi ? multi->gl4 : nullptr;
    M.total = M.n[0] + M.n[1];
    unsigned long long mu[3] = {0, 0, 0};
    if (M.total > 0) {
        KG_SOFT_TRY((cudaError_t)mgk.reserve(sizeof(int32_t) * M.total));
        KG_SOFT_TRY((cudaError_t)mgidx.reserve((size_t)MAXG * M.total));
        KG_SOFT_TRY((cudaError_t)mrows.reserve(sizeof(double) * 9 * SOFT_MULTI_ROWS * (size_t)M.total));
        KG_SOFT_TRY((cudaError_t)mused.reserve(sizeof(unsigned long long) * 3));
        KG_SOFT_TRY(cudaMemsetAsync(mused.p, 0, sizeof(unsigned long long) * 3, st));
        M.gk = mgk.as<int32_t>();
        M.gidx = mgidx.as<uint8_t>();
        M.rows = mrows.as<double>();
        soft_multi_site_kernel<<<(unsigned)((M.total + 127) / 128), 128, 0, st>>>(
            M, n_samples, maf, iterations, mgk.as<int32_t>(), mgidx.as<uint8_t>(), mrows.as<double>(),
            mused.as<unsigned long long>());
        KG_SOFT_TRY(cudaGetLastError());
        KG_SOFT_TRY(cudaMemcpyAsync(mu, mused.p, sizeof(mu), cudaMemcpyDeviceToHost, st));
        KG_SOFT_TRY(cudaStreamSynchronize(st));
    }
    if (multi_used)
        for (int k = 0; k < 3; k++) multi_used[k] = (int64_t)mu[k];
    if (nk == 0 && mu[0] + mu[1] + mu[2] == 0) {
        err = "no segregating site left after allele-frequency filtering";
        return KG_ENOSITES;
    }
    const int64_t nk1 = std::max<int64_t>(nk, 1);   // buffers exist even with no biallelic site
    KG_SOFT_TRY((cudaError_t)idx.reserve(sizeof(int32_t) * nk1));
    KG_SOFT_TRY((cudaError_t)kp.reserve(sizeof(double) * nk1));
    KG_SOFT_TRY((cudaError_t)kq.reserve(sizeof(double) * nk1));
    KG_SOFT_TRY((cudaError_t)ctr.reserve(sizeof(unsigned long long) * 6 + sizeof(int)));
    KG_SOFT_TRY(cudaMemcpyAsync(idx.p, ki.data(), sizeof(int32_t) * nk, cudaMemcpyHostToDevice, st));
    KG_SOFT_TRY(cudaMemcpyAsync(kp.p, kpv.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    KG_SOFT_TRY(cudaMemcpyAsync(kq.p, kqv.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    KG_SOFT_TRY(cudaMemsetAsync(ctr.p, 0, sizeof(unsigned long long) * 6 + sizeof(int), st));
    unsigned long long* next = ctr.as<unsigned long long>();
    unsigned long long* stats = next + 1;
    int* no_rows = reinterpret_cast<int*>(next + 6);
    const bool fp64 = precision == KG_PREC_FP64;
    if (!fp64) {
        KG_SOFT_TRY((cudaError_t)g32.reserve(sizeof(float4) * (size_t)(n_samples * nk1)));
        KG_SOFT_TRY((cudaError_t)pq32.reserve(sizeof(float2) * nk1));
        const int64_t total = n_samples * nk;
        if (total > 0) {
            const unsigned blocks = (unsigned)std::min<int64_t>((total + 255) / 256, 148 * 16);
            soft_pack32_kernel<<<blocks, 256, 0, st>>>(gl.as<double>(), n_samples, n_sites, idx.as<int32_t>(),
                                                       kp.as<double>(), kq.as<double>(), nk, g32.as<float4>(),
                                                       pq32.as<float2>());
        }
    }
    const int64_t rows = ns * (ns + 1) / 2;
    int dev = 0, sms = 148;
    KG_SOFT_TRY(cudaGetDevice(&dev));
    KG_SOFT_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int occ = 0;
    KG_SOFT_TRY(cudaFuncSetAttribute(soft_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SOFT_SMEM));
    KG_SOFT_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, soft_pairs_kernel, SOFT_WARPS * 32, SOFT_SMEM));
    const int64_t grid = (int64_t)sms * std::max(1, occ);
    if (M.total > 0) {
        KG_SOFT_TRY((cudaError_t)mscratch.reserve(sizeof(double) * 9 * (size_t)(grid * SOFT_WARPS * M.total)));
        M.scratch = mscratch.as<double>();
    }
    soft_pairs_kernel<<<(unsigned)grid, SOFT_WARPS * 32, SOFT_SMEM, st>>>(
        gl.as<double>(), n_sites, idx.as<int32_t>(), kp.as<double>(), kq.as<double>(), g32.as<float4>(),
        pq32.as<float2>(), fp64 ? 1 : 0, nk, ns, rows, iterations, d_out, next, no_rows, stats, M);
    KG_SOFT_TRY(cudaGetLastError());
    int h_no_rows = 0;
    unsigned long long hs[5] = {0, 0, 0, 0, 0};
    KG_SOFT_TRY(cudaMemcpyAsync(&h_no_rows, no_rows, sizeof(int), cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaMemcpyAsync(hs, stats, sizeof(hs), cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaStreamSynchronize(st));
    if (counters)
        for (int i = 0; i < 5; i++) counters[i] = hs[i];
    if (h_no_rows) {
        err = "a pair shares no called segregating site";
        return KG_ENOSITES;
    }
    return KG_OK;
}

}  // namespace kg
