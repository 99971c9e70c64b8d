// kg_pair.cuh — the all-pairs maximum-likelihood Jacquard estimator on sm_100a.
//
// One warp owns one pair (x, y) at a time and takes the next from a device
// work queue (an atomic counter) when its SQP finishes, so pairs that converge
// in few iterations free their warp at once.
//
// Per pair, the jointly observed segregating sites are first sorted once by
// genotype-pair *shape* into per-warp scratch lists (segments of 2048 sites).
// The nine one-hot likelihood rows of the reference (src/mixture.rs:96-236)
// fall into five shapes, each a monomial vector in the site's allele
// frequency t (and w = p q):
//   A  (0/0,0/0) (1/1,1/1): L = [t, t^2, t^2, t^3, t^2, t^3, t^2, t^3, t^4]
//   B1 (hom, het):          L = w [0,0,1,2t,0,0,0,t,2t^2]      t = freq of x's allele
//   B2 (het, hom):          L = w [0,0,0,0,1,2t,0,t,2t^2]      t = freq of y's allele
//   C  (hom, other hom):    L = w [0,1,0,ty,0,tx,0,0,w]
//   D  (het, het):          L = w [0,0,0,0,0,0,2,1,4w]
// so every SQP pass streams shape-uniform lists and accumulates per-shape
// moments (sum r t^k, sum r^2 t^k, ...) instead of the dense 9 + 45 sums of
// src/jacquard/grad_hess.rs:44-449; g and H are rebuilt from the 45 moments in
// FP64.  f = -(1/n) sum log(eps + L.D), g = -(1/n) sum L r, H = (1/n) sum L L' r^2
// with r = 1/(eps + L.D) (src/jacquard/objective.rs:9-20, grad_hess.rs:13-41).
//
// Precision (KG_PREC_FP32C): per-site terms in FP32 with MUFU rcp/lg2 (one lg2
// per four sites), the pair's coefficients split hi+lo so the evaluation point
// is the exact FP64 iterate, FP32 partial sums promoted to FP64 per segment, and
// near convergence the objective change is summed directly as
// log(d_new/d_old) = -log1p(-delta/d_new) so the Armijo test (src/sqp.rs:294)
// keeps its resolution.  The 9x9 QP, LDL^T, KKT and condition estimate are
// FP64.  Pairs whose condition estimate is large, or whose FP32 KKT residual
// stalls, are re-evaluated with FP64 passes.
#pragma once

#include <cstdint>
#include <math_constants.h>

#include "kestrel_gpu.h"
#include "kg_rowsolve.cuh"
#include "kg_solver.cuh"

namespace kg {

constexpr int SEG_SITES = 2048;             // padding unit of the bit planes
constexpr int SEG_WORDS = SEG_SITES / 32;   // 32-site plane words per padding unit
constexpr int UNIT_SITES = 1024;            // sites per sort unit (one plane word per lane)
constexpr int UNIT_WORDS = UNIT_SITES / 32;

// Position of kept site k in the unit-transposed frequency arrays: site
// 1024 u + 32 l + i (lane l's word, bit i) sits at 1024 u + 32 i + l, so the
// lanes of a warp stepping through bit i of their words read 32 consecutive
// values.
__host__ __device__ __forceinline__ int64_t freq_index(int64_t k) {
    return (k & ~(int64_t)(UNIT_SITES - 1)) | ((k & 31) << 5) | ((k >> 5) & 31);
}

enum : int { COHORT_TRIANGLE = 0, COHORT_RECT = 1 };

// Device-side description of one cohort (or one serving request).
struct CohortDev {
    const uint2* planes_x;   // [rows_x][plane_stride] {lo, hi} bit planes of 32 sites
    const uint2* planes_y;   // [rows_y][plane_stride] (== planes_x for a triangle)
    int64_t plane_stride;    // words per row (multiple of SEG_WORDS)
    const float* p32;        // REF frequency per kept site in FP32, padded, unit-transposed (freq_index)
    const double* p64;       // REF frequency per kept site, padded, unit-transposed (freq_index)
    const double* q64;       // ALT frequency per kept site, padded
    int32_t n_sites;         // kept (segregating) sites
    int32_t n_units;         // sort units of UNIT_SITES kept sites
    int32_t kind;            // COHORT_TRIANGLE or COHORT_RECT
    int32_t method;          // ESTIMATOR_ML or ESTIMATOR_CLS
    int64_t n_x;             // triangle: num_samples; rect: query rows
    int64_t n_y;             // rect: panel rows
    int64_t pair_begin;      // first global work index
    int64_t n_pairs;
    kg_output* out;          // rows in the reference's order
    uint64_t max_iter;       // SQP iteration limit of this cohort's pairs (CLS: QP iterations)
    const double* cls_q;     // CLS: the 9 x 9 quadratic matrix Q (row-major)
    const double* cls_cmulti;  // CLS: per output row, the 9 summed rows of its tri-/tetra-allelic sites (or NULL)
    double cls_m;            // CLS: the sites M that Q and c are divided by (biallelic + multi-allelic)
    // ML: tri- and tetra-allelic sites (triangle cohorts; ml_nk = 0 otherwise)
    const uint8_t* ml_gr;    // [samples][ml_stride] reduced genotype, ML_ZERO_ROW or ML_MISSING
    const uint32_t* ml_obs;  // [samples][ml_stride / 32] called bits
    const int2* ml_site;     // per kept site: {first row, reduced genotypes G'}
    const double* ml_rows;   // [rows][9] m[g'x][g'y]
    const float4* ml_rows32; // [rows][3] the same rows in FP32 (9 values and 3 zeros)
    int32_t ml_nk;           // kept sites
    int32_t ml_stride;       // bytes per sample row of ml_gr (a multiple of 32)
};

// Reduced genotype codes of the ML path's tri- and tetra-allelic sites: a call
// that uses a dropped allele (its likelihood row becomes all zeros) and a
// missing call.
constexpr uint8_t ML_ZERO_ROW = 0xFE;
constexpr uint8_t ML_MISSING = 0xFF;

// The estimators: maximum likelihood (the GL/PL path, src/coefficients.rs:40-141)
// and the hard-call conditional least squares with the Brier objective (the
// reference's default -f GT, src/coefficients.rs:166-278).
enum : int { ESTIMATOR_ML = 0, ESTIMATOR_CLS = 1 };

// The two alleles (i <= j) of a genotype index in the VCF order, j (j + 1) / 2 + i
// (src/coefficients.rs:19-38); indices 0..9 cover up to four alleles.
__host__ __device__ inline void genotype_alleles(int g, int& i, int& j) {
    j = g >= 6 ? 3 : g >= 3 ? 2 : g >= 1 ? 1 : 0;
    i = g - j * (j + 1) / 2;
}

// m[gx][gy] of a site with any number of alleles (frequencies f): the nine
// conditional probabilities of the joint genotypes (i, j), (k, l) given each
// Jacquard state, the table of src/iis.rs:279-462, evaluated from its
// definition: every ordering of each unordered genotype (x1 x2 = a1 a2, y1 y2 =
// b1 b2) adds, per state, the product over the state's identity classes of the
// class's allele frequency, when all of a class's members carry one allele.
// Classes: 1 {x1 x2 y1 y2}; 2 {x1 x2}{y1 y2}; 3 {x1 x2 y1}{y2}; 4 {x1 x2}{y1}{y2};
// 5 {x1 y1 y2}{x2}; 6 {y1 y2}{x1}{x2}; 7 {x1 y1}{x2 y2}; 8 {x1 y1}{x2}{y2};
// 9 all apart.
__host__ __device__ inline void iis_row(int i, int j, int k, int l, double f0, double f1, double f2, double f3,
                                        double* row) {
    // frequencies by allele without an indexed array (registers, not local memory)
    auto F = [=](int a) { return a == 0 ? f0 : a == 1 ? f1 : a == 2 ? f2 : f3; };
#pragma unroll
    for (int s = 0; s < 9; s++) row[s] = 0.0;
    const int nx = i == j ? 1 : 2, ny = k == l ? 1 : 2;
    for (int u = 0; u < nx; u++) {
        const int a1 = u ? j : i, a2 = u ? i : j;
        const double fa1 = F(a1), fa2 = F(a2);
        for (int w = 0; w < ny; w++) {
            const int b1 = w ? l : k, b2 = w ? k : l;
            const double fb1 = F(b1), fb2 = F(b2);
            const bool xx = a1 == a2, yy = b1 == b2, s1 = a1 == b1, s2 = a2 == b2;
            const double xy = fa1 * fa2;
            if (xx && yy && s1) row[0] += fa1;
            if (xx && yy) row[1] += fa1 * fb1;
            if (xx && s1) row[2] += fa1 * fb2;
            if (xx) row[3] += fa1 * fb1 * fb2;
            if (yy && s1) row[4] += fb1 * fa2;
            if (yy) row[5] += fb1 * xy;
            if (s1 && s2) row[6] += xy;
            if (s1) row[7] += xy * fb2;
            row[8] += xy * fb1 * fb2;
        }
    }
}

// m[gx][gy] of one biallelic site for the CLS estimator: src/iis.rs:279-462
// with the biallelic joint-genotype modes of src/conditional.rs:6-55 (allele 0
// = REF with frequency p, allele 1 = ALT with q), products in the reference's
// order.
__host__ __device__ inline void cls_row(int gx, int gy, double p, double q, double* row) {
    for (int k = 0; k < 9; k++) row[k] = 0.0;
    switch (gx * 3 + gy) {
    case 0: case 8: {   // ii-ii
        const double pi = gx == 0 ? p : q, pi2 = pi * pi, pi3 = pi2 * pi;
        row[0] = pi; row[1] = pi2; row[2] = pi2; row[3] = pi3; row[4] = pi2;
        row[5] = pi3; row[6] = pi2; row[7] = pi3; row[8] = pi2 * pi2;
        break;
    }
    case 2: case 6: {   // ii-kk
        const double pi = gx == 0 ? p : q, pk = gx == 0 ? q : p, pi2 = pi * pi, pk2 = pk * pk;
        row[1] = pi * pk; row[3] = pi * pk2; row[5] = pi2 * pk; row[8] = pi2 * pk2;
        break;
    }
    case 1: case 7: {   // ii-il (0/0, 0/1) and ii-ki (1/1, 0/1)
        const double pi = gx == 0 ? p : q, po = gx == 0 ? q : p, pi2 = pi * pi, pi3 = pi2 * pi;
        row[2] = pi * po; row[3] = (2.0 * pi2) * po; row[7] = pi2 * po; row[8] = (2.0 * pi3) * po;
        break;
    }
    case 3: {           // ij-ii
        const double pi2 = p * p, pi3 = pi2 * p;
        row[4] = p * q; row[5] = (2.0 * pi2) * q; row[7] = pi2 * q; row[8] = (2.0 * pi3) * q;
        break;
    }
    case 5: {           // ij-jj
        const double pj2 = q * q;
        row[4] = p * q; row[5] = (2.0 * pj2) * p; row[7] = pj2 * p; row[8] = (2.0 * (pj2 * q)) * p;
        break;
    }
    case 4: {           // ij-ij
        row[6] = (2.0 * p) * q; row[7] = (p * q) * (p + q); row[8] = (4.0 * (p * p)) * (q * q);
        break;
    }
    }
}

struct RunCounters {
    unsigned long long gh_passes;
    unsigned long long obj_passes;
    unsigned long long fp64_passes;
    unsigned long long fp64_pairs;
    unsigned long long pair_sites;
    unsigned long long work_units;
    unsigned long long nosite_pairs;
    unsigned long long nonconverged;
    unsigned long long flops_fp32;
    unsigned long long flops_fp64;
    unsigned long long shape_sites[5];
    unsigned long long cycles[5];   // SM clocks per phase: count, scatter, site passes, solver, streams
    unsigned long long stalled_waits;   // device waits that ran out of their limit
};

struct PairLaunch {
    const CohortDev* cohorts;
    int n_cohorts;
    int precision;               // 0 FP32C, 1 FP64
    int64_t total_pairs;
    unsigned long long* queue;   // next work index
    double* lists;               // per warp: the pair's shape lists (FP32 or FP64 values)
    int64_t list_stride;         // 8-byte words per warp
    Tune tune;
    RunCounters* counters;
};

// ------------------------------------------------------------ FP32 helpers

// MUFU reciprocal: at most 1 ulp from 1 / d over the whole FP32 range.
__device__ __forceinline__ float rcp_approx(float d) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
    return r;
}

__device__ __forceinline__ float lg2_approx(float a) {
    float r;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

// log(d_new / d_old) with d_old = d_new - delta, given z = delta / d_new:
// -log(1 - z).  Taylor series (sum z^k / k, k <= 6) for |z| <= 1/16, whose
// truncation error is below 1e-8 relative; the MUFU log2 otherwise.
__device__ __forceinline__ float neg_log1m(float z) {
    if (fabsf(z) <= 0.0625f) {
        float s = fmaf(z, 0.16666667f, 0.2f);
        s = fmaf(z, s, 0.25f);
        s = fmaf(z, s, 0.33333334f);
        s = fmaf(z, s, 0.5f);
        s = fmaf(z, s, 1.0f);
        return z * s;
    }
    return -0.6931472f * lg2_approx(1.0f - z);
}

struct HiLo {
    float h, l;
};

__device__ __forceinline__ HiLo split(double v) {
    HiLo r;
    r.h = (float)v;
    r.l = (float)(v - (double)r.h);
    return r;
}

// Moment sums, in the order used by the rebuild:
//  0..3  GA  sum r t^k, k=1..4          4..10 HA  sum r^2 t^k, k=2..8
// 11..13 GB1 sum r w t^k, k=0..2        14..18 HB1 sum r^2 w^2 t^k, k=0..4
// 19..21 GB2                            22..26 HB2
// 27..30 GC  sum r w {1,ty,tx,w}        31..39 HC sum r^2 w^2 {1,ty,tx,w,ty^2,tx^2,w ty,w tx,w^2}
// 40..41 GD  sum r w {1,w}              42..44 HD  sum r^2 w^2 {1,w,w^2}
constexpr int NMOM = 45;


// Per-pass coefficients of L.D for each shape (see the header comment).
struct PassCoef {
    // FP64 values
    double a[4];     // A: t (a1 + t (a2 + t (a3 + t a4)))
    double b1[3];    // B1: w (b0 + t (b1 + t b2))
    double b2[3];    // B2
    double c[4];     // C: w (c0 + ty c1 + tx c2 + w c3)
    double d[2];     // D: w (d0 + w d1)
};

__device__ __forceinline__ void make_coef(const double* D, PassCoef& k) {
    k.a[0] = D[0];
    k.a[1] = D[1] + D[2] + D[4] + D[6];
    k.a[2] = D[3] + D[5] + D[7];
    k.a[3] = D[8];
    k.b1[0] = D[2];
    k.b1[1] = 2.0 * D[3] + D[7];
    k.b1[2] = 2.0 * D[8];
    k.b2[0] = D[4];
    k.b2[1] = 2.0 * D[5] + D[7];
    k.b2[2] = 2.0 * D[8];
    k.c[0] = D[1];
    k.c[1] = D[3];
    k.c[2] = D[5];
    k.c[3] = D[8];
    k.d[0] = 2.0 * D[6] + D[7];
    k.d[1] = 4.0 * D[8];
}

// Rebuilds S = sum L r (9) and T = sum L L' r^2 (9x9, symmetric) from moments.
__device__ inline void rebuild(const double* m, double* S, double* T) {
    const int e[9] = {1, 2, 2, 3, 2, 3, 2, 3, 4};
    for (int i = 0; i < 9; i++) S[i] = m[0 + e[i] - 1];
    for (int i = 0; i < 9; i++)
        for (int j = 0; j < 9; j++) T[i * 9 + j] = m[4 + e[i] + e[j] - 2];
    // B1 on {2,3,7,8} and B2 on {4,5,7,8}: coefficient {1,2,1,2}, power {0,1,1,2}
    const int cb[4] = {1, 2, 1, 2};
    const int pb[4] = {0, 1, 1, 2};
    const int i1[4] = {2, 3, 7, 8};
    const int i2[4] = {4, 5, 7, 8};
    for (int a = 0; a < 4; a++) {
        S[i1[a]] += cb[a] * m[11 + pb[a]];
        S[i2[a]] += cb[a] * m[19 + pb[a]];
        for (int b = 0; b < 4; b++) {
            double c = (double)(cb[a] * cb[b]);
            T[i1[a] * 9 + i1[b]] += c * m[14 + pb[a] + pb[b]];
            T[i2[a] * 9 + i2[b]] += c * m[22 + pb[a] + pb[b]];
        }
    }
    // C on {1,3,5,8} with monomials {1, ty, tx, w}
    S[1] += m[27];
    S[3] += m[28];
    S[5] += m[29];
    S[8] += m[30];
    const int ic[4] = {1, 3, 5, 8};
    // product table of {1,ty,tx,w} -> HC index (31 + k)
    const int hc[4][4] = {{0, 1, 2, 3}, {1, 4, 3, 6}, {2, 3, 5, 7}, {3, 6, 7, 8}};
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) T[ic[a] * 9 + ic[b]] += m[31 + hc[a][b]];
    // D on {6,7,8}: L = w [2, 1, 4w]
    S[6] += 2.0 * m[40];
    S[7] += m[40];
    S[8] += 4.0 * m[41];
    const int id[3] = {6, 7, 8};
    const double cd[3] = {2.0, 1.0, 4.0};
    const int pd[3] = {0, 0, 1};
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) T[id[a] * 9 + id[b]] += cd[a] * cd[b] * m[42 + pd[a] + pd[b]];
}

// ------------------------------------------------------------- sorting

// Shape masks of 32 sites from the {lo, hi} planes of x and y (code = 2 hi + lo;
// 3 = missing, which is neither hom nor het).  sel picks t = ALT frequency:
// x's allele for A, B1 and C; y's allele for B2.
struct ShapeMasks {
    uint32_t m[5];
    uint32_t sel;
};

__device__ __forceinline__ ShapeMasks shape_masks(uint2 X, uint2 Y) {
    ShapeMasks r;
    uint32_t xhom = ~X.x, xhet = X.x & ~X.y;
    uint32_t yhom = ~Y.x, yhet = Y.x & ~Y.y;
    uint32_t same = ~(X.y ^ Y.y);
    r.m[0] = xhom & yhom & same;   // A
    r.m[1] = xhom & yhet;          // B1
    r.m[2] = xhet & yhom;          // B2
    r.m[3] = xhom & yhom & ~same;  // C
    r.m[4] = xhet & yhet;          // D
    r.sel = (X.y & ~r.m[2]) | (Y.y & r.m[2]);
    return r;
}

__host__ __device__ __forceinline__ int64_t align4(int64_t v) { return (v + 3) & ~(int64_t)3; }

// Per-pair list layout: shape s occupies [start[s], start[s] + cnt[s]) elements
// of the warp's list buffer; starts are multiples of 4 (16-byte float4 loads).
struct PairLists {
    int64_t start[5];
    int64_t cnt[5];
    int64_t n;
};

__device__ inline void count_shapes(const CohortDev& co, int64_t x, int64_t y, int lane, PairLists& pl) {
    const uint2* px = co.planes_x + x * co.plane_stride;
    const uint2* py = co.planes_y + y * co.plane_stride;
    unsigned c[5] = {0, 0, 0, 0, 0};
    const int nw = co.n_units * UNIT_WORDS;
    for (int w = lane; w < nw; w += 32) {
        ShapeMasks sm = shape_masks(px[w], py[w]);
#pragma unroll
        for (int s = 0; s < 5; s++) c[s] += __popc(sm.m[s]);
    }
    int64_t st = 0;
    pl.n = 0;
#pragma unroll
    for (int s = 0; s < 5; s++) {
        unsigned v = c[s];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        pl.cnt[s] = v;
        pl.start[s] = st;
        st = align4(st + v);
        pl.n += v;
    }
}

// Writes the frequency value t of every jointly observed site into its shape
// list (in FP32 or FP64), one unit of 1024 sites at a time.  The unit's REF
// frequencies are first staged in shared memory with coalesced loads (lane l
// holds sites 32 l .. 32 l + 31, stored transposed so the per-site reads are
// conflict-free); t is p or 1 - p by the site's sel bit.  FP32 values go through
// a shared output buffer so the global stores stay coalesced; FP64 values (the
// FP64 form and re-evaluated pairs) are stored directly.
// scatter_units covers units [u0, u1) with the shapes' write positions starting
// at off[]; scatter_shapes is the whole pair.
template <class T>
__device__ inline void scatter_units(const CohortDev& co, int64_t x, int64_t y, int lane, int u0,
                                     int u1, const int64_t* off0, T* lists, char* wsm) {
    const uint2* px = co.planes_x + x * co.plane_stride;
    const uint2* py = co.planes_y + y * co.plane_stride;
    T* stage = reinterpret_cast<T*>(wsm);                       // UNIT_SITES values
    float* obuf = reinterpret_cast<float*>(wsm + UNIT_SITES * sizeof(float));  // FP32 only
    int64_t off[5];
#pragma unroll
    for (int s = 0; s < 5; s++) off[s] = off0[s];
    for (int u = u0; u < u1; u++) {
        const int w = u * UNIT_WORDS + lane;
        const uint2 X = px[w], Y = py[w];
        // stage the unit's REF frequencies (already unit-transposed: site
        // 32 lane + i at [i * 32 + lane])
        if (sizeof(T) == 4) {
            const float4* src = reinterpret_cast<const float4*>(co.p32 + (int64_t)u * UNIT_SITES);
#pragma unroll
            for (int v4 = 0; v4 < 8; v4++) reinterpret_cast<float4*>(stage)[v4 * 32 + lane] = src[v4 * 32 + lane];
        } else {
            const double2* src = reinterpret_cast<const double2*>(co.p64 + (int64_t)u * UNIT_SITES);
#pragma unroll
            for (int v2 = 0; v2 < 16; v2++) reinterpret_cast<double2*>(stage)[v2 * 32 + lane] = src[v2 * 32 + lane];
        }
        ShapeMasks sm = shape_masks(X, Y);
        unsigned long long v = 0;
#pragma unroll
        for (int s = 0; s < 5; s++) v |= (unsigned long long)__popc(sm.m[s]) << (11 * s);
        unsigned long long inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        const unsigned long long tot = __shfl_sync(0xffffffffu, inc, 31);
        const unsigned long long exc = inc - v;
        unsigned ustart[6];
        ustart[0] = 0;
#pragma unroll
        for (int s = 0; s < 5; s++) ustart[s + 1] = ustart[s] + (unsigned)((tot >> (11 * s)) & 0x7FF);
        __syncwarp();
#pragma unroll
        for (int s = 0; s < 5; s++) {
            unsigned rank = (unsigned)((exc >> (11 * s)) & 0x7FF);
            uint32_t mm = sm.m[s];
            while (mm) {
                const int i = __ffs(mm) - 1;
                mm &= mm - 1;
                const T p = stage[i * 32 + lane];
                const T t = ((sm.sel >> i) & 1u) ? (T)1 - p : p;
                if (sizeof(T) == 4) obuf[ustart[s] + rank] = (float)t;
                else lists[off[s] + rank] = t;
                rank++;
            }
        }
        __syncwarp();
        if (sizeof(T) == 4) {
#pragma unroll
            for (int s = 0; s < 5; s++) {
                const unsigned ns = ustart[s + 1] - ustart[s];
                float* dst = reinterpret_cast<float*>(lists) + off[s];
                const float* srcb = obuf + ustart[s];
                for (unsigned j = lane; j < ns; j += 32) dst[j] = srcb[j];
            }
            __syncwarp();
        }
#pragma unroll
        for (int s = 0; s < 5; s++) off[s] += ustart[s + 1] - ustart[s];
    }
}

template <class T>
__device__ inline void scatter_shapes(const CohortDev& co, int64_t x, int64_t y, int lane,
                                      const PairLists& pl, T* lists, char* wsm) {
    scatter_units<T>(co, x, y, lane, 0, co.n_units, pl.start, lists, wsm);
}

// ----------------------------------------------------------- FP32 passes

// Warp-uniform pass coefficients, kept in shared memory and read at the top
// of each shape's stream so only that shape's values occupy registers.
struct Coef32 {
    HiLo a[4], b1[3], b2[3], c[4], d[2];
    float sa[4], sb1[3], sb2[3], sc[4], sd[2];  // step coefficients (OBJ_DIFF)
};

constexpr int WARP_SMEM_BUF = UNIT_SITES * 8;   // frequency stage + FP32 output buffer
constexpr int WARP_SMEM_COEF = 256;
constexpr int WARP_SMEM = WARP_SMEM_BUF + WARP_SMEM_COEF;
static_assert(sizeof(Coef32) <= WARP_SMEM_COEF, "coefficients must fit");

template <class T>
__device__ __forceinline__ T ld_volatile(const T* p) { return *reinterpret_cast<const volatile T*>(p); }

__device__ __forceinline__ HiLo ldk(const HiLo* p) {
    HiLo r;
    r.h = ld_volatile(&p->h);
    r.l = ld_volatile(&p->l);
    return r;
}

// Per-lane FP64 sums of one pass: NMOM moments + the objective term.
struct LaneSums {
    double m[NMOM];
    double obj;
};

constexpr int HESS_FLUSH = 8;   // loop iterations (8 sites each) between FP32 -> FP64 Hessian flushes

// The FP32 closed form of one shape: coefficients of the pending pass (from
// shared memory) and the per-site update of the FP32 partial sums.  The
// moments share their products: with u = r c (c = t for A, w otherwise) the
// gradient terms are u times the shape's monomials (each summed by one FMA,
// a single rounding) and every Hessian term is a product of two of them.
//
// LO = true evaluates L.Delta with the hi + lo split coefficients (the FP64
// iterate to ~1e-14); LO = false uses the hi parts only, and the solve step
// restores the lo part to first order in FP64 from the moments themselves
// (lo_correction), which leaves an error of (lo / hi)^2 ~ 1e-15 relative.
template <int S, bool LO = true>
struct Shape32 {
    static constexpr int NG = S == 0 ? 4 : S == 3 ? 4 : S == 4 ? 2 : 3;
    static constexpr int NH = S == 0 ? 7 : S == 3 ? 9 : S == 4 ? 3 : 5;
    static constexpr int GOFF = S == 0 ? 0 : S == 1 ? 11 : S == 2 ? 19 : S == 3 ? 27 : 40;
    static constexpr int HOFF = GOFF + NG;
    HiLo k0, k1, k2, k3;
    float s0, s1, s2, s3;
    bool diff;

    __device__ __forceinline__ void load(const Coef32* K, bool diff_) {
        diff = diff_;
        s0 = s1 = s2 = s3 = 0.f;
        if (S == 0) { k0 = ldk(&K->a[0]); k1 = ldk(&K->a[1]); k2 = ldk(&K->a[2]); k3 = ldk(&K->a[3]); }
        if (S == 1) { k0 = ldk(&K->b1[0]); k1 = ldk(&K->b1[1]); k2 = ldk(&K->b1[2]); k3 = HiLo{0.f, 0.f}; }
        if (S == 2) { k0 = ldk(&K->b2[0]); k1 = ldk(&K->b2[1]); k2 = ldk(&K->b2[2]); k3 = HiLo{0.f, 0.f}; }
        if (S == 3) { k0 = ldk(&K->c[0]); k1 = ldk(&K->c[1]); k2 = ldk(&K->c[2]); k3 = ldk(&K->c[3]); }
        if (S == 4) { k0 = ldk(&K->d[0]); k1 = ldk(&K->d[1]); k2 = HiLo{0.f, 0.f}; k3 = HiLo{0.f, 0.f}; }
        if (diff) {
            const float* sp = S == 0 ? K->sa : S == 1 ? K->sb1 : S == 2 ? K->sb2 : S == 3 ? K->sc : K->sd;
            s0 = ld_volatile(&sp[0]);
            s1 = ld_volatile(&sp[1]);
            if (S != 4) s2 = ld_volatile(&sp[2]);
            if (S == 0 || S == 3) s3 = ld_volatile(&sp[3]);
        }
    }

    // one site's gradient and Hessian terms into the FP32 partials g and h;
    // returns d = L.Delta + eps, r = 1 / d and the site's scale c (t for A,
    // w for B, C, D)
    __device__ __forceinline__ void core(float t, float* g, float* h, float& d, float& r, float& c) const {
        const float EPS = 1e-8f;
        if (S == 0) {
            float ph = fmaf(fmaf(fmaf(k3.h, t, k2.h), t, k1.h), t, k0.h);
            if (LO) ph = ph + fmaf(fmaf(fmaf(k3.l, t, k2.l), t, k1.l), t, k0.l);
            d = fmaf(t, ph, EPS);
            r = rcp_approx(d);
            const float u = r * t, v1 = u * t, v2 = v1 * t, v3 = v2 * t;   // r t^1..4
            g[0] += u; g[1] = fmaf(u, t, g[1]); g[2] = fmaf(v1, t, g[2]); g[3] = fmaf(v2, t, g[3]);
            h[0] = fmaf(u, u, h[0]); h[1] = fmaf(u, v1, h[1]); h[2] = fmaf(v1, v1, h[2]);
            h[3] = fmaf(v1, v2, h[3]); h[4] = fmaf(v2, v2, h[4]); h[5] = fmaf(v2, v3, h[5]);
            h[6] = fmaf(v3, v3, h[6]);
            c = t;
        } else if (S == 1 || S == 2) {
            const float w = fmaf(-t, t, t);
            float ph = fmaf(fmaf(k2.h, t, k1.h), t, k0.h);
            if (LO) ph = ph + fmaf(fmaf(k2.l, t, k1.l), t, k0.l);
            d = fmaf(w, ph, EPS);
            r = rcp_approx(d);
            const float v = r * w, v1 = v * t, v2 = v1 * t;                 // r w t^0..2
            g[0] += v; g[1] = fmaf(v, t, g[1]); g[2] = fmaf(v1, t, g[2]);
            h[0] = fmaf(v, v, h[0]); h[1] = fmaf(v, v1, h[1]); h[2] = fmaf(v1, v1, h[2]);
            h[3] = fmaf(v1, v2, h[3]); h[4] = fmaf(v2, v2, h[4]);
            c = w;
        } else if (S == 3) {
            const float ty = 1.0f - t;   // t = tx, the frequency of x's allele
            const float w = t * ty;
            float ph = fmaf(w, k3.h, fmaf(t, k2.h, fmaf(ty, k1.h, k0.h)));
            if (LO) ph = ph + fmaf(w, k3.l, fmaf(t, k2.l, fmaf(ty, k1.l, k0.l)));
            d = fmaf(w, ph, EPS);
            r = rcp_approx(d);
            const float v = r * w, a = v * ty, b = v * t, e = v * w;          // r w {1, ty, t, w}
            g[0] += v; g[1] = fmaf(v, ty, g[1]); g[2] = fmaf(v, t, g[2]); g[3] = fmaf(v, w, g[3]);
            h[0] = fmaf(v, v, h[0]); h[1] = fmaf(v, a, h[1]); h[2] = fmaf(v, b, h[2]);
            h[3] = fmaf(v, e, h[3]); h[4] = fmaf(a, a, h[4]); h[5] = fmaf(b, b, h[5]);
            h[6] = fmaf(e, a, h[6]); h[7] = fmaf(e, b, h[7]); h[8] = fmaf(e, e, h[8]);
            c = w;
        } else {
            const float w = fmaf(-t, t, t);
            float ph = fmaf(w, k1.h, k0.h);
            if (LO) ph = ph + fmaf(w, k1.l, k0.l);
            d = fmaf(w, ph, EPS);
            r = rcp_approx(d);
            const float v = r * w, a = v * w;                                // r w {1, w}
            g[0] += v; g[1] = fmaf(v, w, g[1]);
            h[0] = fmaf(v, v, h[0]); h[1] = fmaf(v, a, h[1]); h[2] = fmaf(a, a, h[2]);
            c = w;
        }
    }

    // the site's objective term in diff mode: -log(1 - delta / d_new)
    __device__ __forceinline__ float diff_term(float t, float r, float c) const {
        float dl;
        if (S == 0) dl = t * fmaf(fmaf(fmaf(s3, t, s2), t, s1), t, s0);
        else if (S == 1 || S == 2) dl = c * fmaf(fmaf(s2, t, s1), t, s0);
        else if (S == 3) dl = c * fmaf(c, s3, fmaf(t, s2, fmaf(1.0f - t, s1, s0)));
        else dl = c * fmaf(c, s1, s0);
        return neg_log1m(dl * r);
    }

    // one site: adds into the FP32 partials g, ob (per iteration) and h
    __device__ __forceinline__ void site(float t, float* g, float& ob, float* h) const {
        float d, r, c;
        core(t, g, h, d, r, c);
        if (!diff) ob += lg2_approx(d);
        else ob += diff_term(t, r, c);
    }

    // four sites (one float4), the objective kind fixed at compile time: in
    // direct mode one lg2 of the product of the four d (each d lies in
    // [1e-8, 1 + 1e-8], so the product stays a normal FP32 number)
    template <bool DIFF>
    __device__ __forceinline__ void site4(float4 v, float* g, float& ob, float* h) const {
        float d0, d1, d2, d3, r0, r1, r2, r3, c0, c1, c2, c3;
        core(v.x, g, h, d0, r0, c0);
        core(v.y, g, h, d1, r1, c1);
        core(v.z, g, h, d2, r2, c2);
        core(v.w, g, h, d3, r3, c3);
        if (!DIFF) {
            ob += lg2_approx((d0 * d1) * (d2 * d3));
        } else {
            ob += diff_term(v.x, r0, c0);
            ob += diff_term(v.y, r1, c1);
            ob += diff_term(v.z, r2, c2);
            ob += diff_term(v.w, r3, c3);
        }
    }
};

// eps + L.x over nine entries as three interleaved chains (five dependent
// operations instead of nine), for the generic-row evaluations
__device__ __forceinline__ float dot9_eps(const float* L, const float* x, float eps) {
    const float a = fmaf(L[0], x[0], fmaf(L[3], x[3], fmaf(L[6], x[6], eps)));
    const float b = fmaf(L[1], x[1], fmaf(L[4], x[4], L[7] * x[7]));
    const float c = fmaf(L[2], x[2], fmaf(L[5], x[5], L[8] * x[8]));
    return a + (b + c);
}

// ---------------------------------------------------------------- packed pairs
// Shape32's hi-coefficient site arithmetic on two sites at once with the
// sm_100 packed FP32 instructions (fma/mul/add .f32x2): one instruction per
// operation for both sites, each half rounded exactly as the scalar operation
// (the reciprocal and the logarithm stay scalar MUFU operations).  Gradient,
// Hessian and objective partials are pairs, one half per site parity.

__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 rcp2(float2 d) { return make_float2(rcp_approx(d.x), rcp_approx(d.y)); }

template <int S>
struct Shape32x2 {
    using One = Shape32<S, false>;
    static constexpr int NG = One::NG, NH = One::NH, GOFF = One::GOFF, HOFF = One::HOFF;
    float2 k0, k1, k2, k3, s0, s1, s2, s3;

    __device__ __forceinline__ void load(const Coef32* K, bool diff) {
        const HiLo* kk = S == 0 ? K->a : S == 1 ? K->b1 : S == 2 ? K->b2 : S == 3 ? K->c : K->d;
        k0 = dup2(ld_volatile(&kk[0].h));
        k1 = dup2(ld_volatile(&kk[1].h));
        k2 = S == 4 ? dup2(0.f) : dup2(ld_volatile(&kk[2].h));
        k3 = (S == 0 || S == 3) ? dup2(ld_volatile(&kk[3].h)) : dup2(0.f);
        s0 = s1 = s2 = s3 = dup2(0.f);
        if (diff) {
            const float* sp = S == 0 ? K->sa : S == 1 ? K->sb1 : S == 2 ? K->sb2 : S == 3 ? K->sc : K->sd;
            s0 = dup2(ld_volatile(&sp[0]));
            s1 = dup2(ld_volatile(&sp[1]));
            if (S != 4) s2 = dup2(ld_volatile(&sp[2]));
            if (S == 0 || S == 3) s3 = dup2(ld_volatile(&sp[3]));
        }
    }

    // Shape32::core on a pair of sites
    __device__ __forceinline__ void core(float2 t, float2* g, float2* h, float2& d, float2& r, float2& c) const {
        const float2 EPS = dup2(1e-8f);
        if (S == 0) {
            const float2 ph = fma2(fma2(fma2(k3, t, k2), t, k1), t, k0);
            d = fma2(t, ph, EPS);
            r = rcp2(d);
            const float2 u = mul2(r, t), v1 = mul2(u, t), v2 = mul2(v1, t), v3 = mul2(v2, t);
            g[0] = add2(g[0], u); g[1] = fma2(u, t, g[1]); g[2] = fma2(v1, t, g[2]); g[3] = fma2(v2, t, g[3]);
            h[0] = fma2(u, u, h[0]); h[1] = fma2(u, v1, h[1]); h[2] = fma2(v1, v1, h[2]);
            h[3] = fma2(v1, v2, h[3]); h[4] = fma2(v2, v2, h[4]); h[5] = fma2(v2, v3, h[5]);
            h[6] = fma2(v3, v3, h[6]);
            c = t;
        } else if (S == 1 || S == 2) {
            const float2 w = fma2(neg2(t), t, t);
            const float2 ph = fma2(fma2(k2, t, k1), t, k0);
            d = fma2(w, ph, EPS);
            r = rcp2(d);
            const float2 v = mul2(r, w), v1 = mul2(v, t), v2 = mul2(v1, t);
            g[0] = add2(g[0], v); g[1] = fma2(v, t, g[1]); g[2] = fma2(v1, t, g[2]);
            h[0] = fma2(v, v, h[0]); h[1] = fma2(v, v1, h[1]); h[2] = fma2(v1, v1, h[2]);
            h[3] = fma2(v1, v2, h[3]); h[4] = fma2(v2, v2, h[4]);
            c = w;
        } else if (S == 3) {
            const float2 ty = add2(dup2(1.0f), neg2(t));
            const float2 w = mul2(t, ty);
            const float2 ph = fma2(w, k3, fma2(t, k2, fma2(ty, k1, k0)));
            d = fma2(w, ph, EPS);
            r = rcp2(d);
            const float2 v = mul2(r, w), a = mul2(v, ty), b = mul2(v, t), e = mul2(v, w);
            g[0] = add2(g[0], v); g[1] = fma2(v, ty, g[1]); g[2] = fma2(v, t, g[2]); g[3] = fma2(v, w, g[3]);
            h[0] = fma2(v, v, h[0]); h[1] = fma2(v, a, h[1]); h[2] = fma2(v, b, h[2]);
            h[3] = fma2(v, e, h[3]); h[4] = fma2(a, a, h[4]); h[5] = fma2(b, b, h[5]);
            h[6] = fma2(e, a, h[6]); h[7] = fma2(e, b, h[7]); h[8] = fma2(e, e, h[8]);
            c = w;
        } else {
            const float2 w = fma2(neg2(t), t, t);
            const float2 ph = fma2(w, k1, k0);
            d = fma2(w, ph, EPS);
            r = rcp2(d);
            const float2 v = mul2(r, w), a = mul2(v, w);
            g[0] = add2(g[0], v); g[1] = fma2(v, w, g[1]);
            h[0] = fma2(v, v, h[0]); h[1] = fma2(v, a, h[1]); h[2] = fma2(a, a, h[2]);
            c = w;
        }
    }

    // z = delta / d_new of Shape32::diff_term on a pair of sites
    __device__ __forceinline__ float2 diff_z(float2 t, float2 r, float2 c) const {
        float2 dl;
        if (S == 0) dl = mul2(t, fma2(fma2(fma2(s3, t, s2), t, s1), t, s0));
        else if (S == 1 || S == 2) dl = mul2(c, fma2(fma2(s2, t, s1), t, s0));
        else if (S == 3) dl = mul2(c, fma2(c, s3, fma2(t, s2, fma2(add2(dup2(1.0f), neg2(t)), s1, s0))));
        else dl = mul2(c, fma2(c, s1, s0));
        return mul2(dl, r);
    }

    // four sites (one float4) as two pairs; o collects the objective terms,
    // one per four sites, in o.y for odd float4 and o.x for even ones, so each
    // half takes every other one.  Direct mode: one lg2 of the product of the
    // four d.  Difference mode: the four terms -log(1 - z_i) as one,
    // -log(1 - w) with 1 - w = prod (1 - z_i), where the w of two sites is
    // z0 + z1 - z0 z1 (no cancellation for small z: w carries the rounding of
    // the z themselves, as the four separate terms would).
    template <bool DIFF>
    __device__ __forceinline__ void site4(float4 v, float2* g, float2& o, float2* h, bool odd) const {
        const float2 ta = make_float2(v.x, v.y), tb = make_float2(v.z, v.w);
        float2 da, db, ra, rb, ca, cb;
        core(ta, g, h, da, ra, ca);
        core(tb, g, h, db, rb, cb);
        float l;
        if (!DIFF) {
            const float2 p = mul2(da, db);
            l = lg2_approx(p.x * p.y);
        } else {
            const float2 za = diff_z(ta, ra, ca), zb = diff_z(tb, rb, cb);
            const float2 w2 = fma2(neg2(za), zb, add2(za, zb));
            l = neg_log1m(fmaf(-w2.x, w2.y, w2.x + w2.y));
        }
        if (odd) o.y += l;
        else o.x += l;
    }
};

// First-order restoration of the lo coefficients for sums taken with the hi
// parts only (Shape32<S, false>).  With d = d_hi + delta, delta = c(t) times
// the lo polynomial, every gradient moment sum_s r c m(s) changes by
// -sum_s r^2 c^2 m(s) lo(s), a combination of the shape's Hessian moments, and
// the natural-log objective by +sum_s delta / d = sum_j lo_j G_j.  mom holds
// the 45 FP64 moments (corrected in place); returns the objective correction.
__device__ inline double lo_correction(double* mom, const Coef32& K) {
    double corr = 0.0;
    // A: G_k = m[k] (r t^{k+1}, k = 0..3), H_m = m[4 + m] (r^2 t^{m+2}); lo = t sum_j l_j t^j
    {
        double l[4], gd[4];
        for (int j = 0; j < 4; j++) l[j] = (double)K.a[j].l;
        for (int k = 0; k < 4; k++) {
            double s = 0.0;
            for (int j = 0; j < 4; j++) s = fma(l[j], mom[4 + k + j], s);
            gd[k] = s;
        }
        for (int j = 0; j < 4; j++) corr = fma(l[j], mom[j], corr);
        for (int k = 0; k < 4; k++) mom[k] -= gd[k];
    }
    // B1, B2: G_k = m[go + k] (r w t^k, k = 0..2), H_m = m[go + 3 + m] (r^2 w^2 t^m)
    for (int b = 0; b < 2; b++) {
        const int go = b == 0 ? 11 : 19;
        const HiLo* kk = b == 0 ? K.b1 : K.b2;
        double l[3], gd[3];
        for (int j = 0; j < 3; j++) l[j] = (double)kk[j].l;
        for (int k = 0; k < 3; k++) {
            double s = 0.0;
            for (int j = 0; j < 3; j++) s = fma(l[j], mom[go + 3 + k + j], s);
            gd[k] = s;
        }
        for (int j = 0; j < 3; j++) corr = fma(l[j], mom[go + j], corr);
        for (int k = 0; k < 3; k++) mom[go + k] -= gd[k];
    }
    // C: G = m[27..30] (r w {1, ty, t, w}), H = m[31..39] (r^2 w^2 {1, ty, t, w, ty^2, t^2, w ty, w t, w^2})
    {
        // products of {1, ty, t, w} x {1, ty, t, w} as Hessian moment indices (ty t = w)
        const int P[4][4] = {{0, 1, 2, 3}, {1, 4, 3, 6}, {2, 3, 5, 7}, {3, 6, 7, 8}};
        double l[4], gd[4];
        for (int j = 0; j < 4; j++) l[j] = (double)K.c[j].l;
        for (int k = 0; k < 4; k++) {
            double s = 0.0;
            for (int j = 0; j < 4; j++) s = fma(l[j], mom[31 + P[k][j]], s);
            gd[k] = s;
        }
        for (int j = 0; j < 4; j++) corr = fma(l[j], mom[27 + j], corr);
        for (int k = 0; k < 4; k++) mom[27 + k] -= gd[k];
    }
    // D: G = m[40..41] (r w {1, w}), H = m[42..44] (r^2 w^2 {1, w, w^2})
    {
        double l[2], gd[2];
        for (int j = 0; j < 2; j++) l[j] = (double)K.d[j].l;
        for (int k = 0; k < 2; k++) {
            double s = 0.0;
            for (int j = 0; j < 2; j++) s = fma(l[j], mom[42 + k + j], s);
            gd[k] = s;
        }
        for (int j = 0; j < 2; j++) corr = fma(l[j], mom[40 + j], corr);
        for (int k = 0; k < 2; k++) mom[40 + k] -= gd[k];
    }
    return corr;
}

// Streams one shape's FP32 list.  Each loop iteration handles two float4
// (8 sites per lane) held in two registers that are refilled right after use,
// so every load has a full iteration to arrive.  Gradient moments and the
// objective are promoted to FP64 every 8 sites, Hessian moments every 64; each
// site is the closed form of its shape (see the file comment).  diff selects
// the log(d_new/d_old) objective.
template <int S>
__device__ __noinline__ void stream32(const float* __restrict__ L, int64_t len, const Coef32* K,
                                      bool diff, int lane, LaneSums& out) {
    using E = Shape32<S>;
    constexpr int NG = E::NG, NH = E::NH, GOFF = E::GOFF, HOFF = E::HOFF;
    E ev;
    ev.load(K, diff);
    double G[NG], H[NH], F = 0.0;
    float h[NH];
#pragma unroll
    for (int i = 0; i < NG; i++) G[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NH; i++) { H[i] = 0.0; h[i] = 0.f; }
    auto site = [&](float t, float* g, float& ob) { ev.site(t, g, ob, h); };

    const int64_t n4 = len >> 2;
    const float4* L4 = reinterpret_cast<const float4*>(L);
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
    int64_t k = lane;
    float4 va = (k < n4) ? L4[k] : z4;
    float4 vb = (k + 32 < n4) ? L4[k + 32] : z4;
    int it = 0;
    while (k < n4) {
        float g[NG], ob = 0.f;
#pragma unroll
        for (int i = 0; i < NG; i++) g[i] = 0.f;
        site(va.x, g, ob);
        site(va.y, g, ob);
        site(va.z, g, ob);
        site(va.w, g, ob);
        va = (k + 64 < n4) ? L4[k + 64] : z4;
        if (k + 32 < n4) {
            site(vb.x, g, ob);
            site(vb.y, g, ob);
            site(vb.z, g, ob);
            site(vb.w, g, ob);
        }
        vb = (k + 96 < n4) ? L4[k + 96] : z4;
#pragma unroll
        for (int i = 0; i < NG; i++) G[i] += (double)g[i];
        F += (double)ob;
        if (++it == HESS_FLUSH) {
#pragma unroll
            for (int i = 0; i < NH; i++) { H[i] += (double)h[i]; h[i] = 0.f; }
            it = 0;
        }
        k += 64;
    }
    if (lane < (int)(len & 3)) {
        float g[NG], ob = 0.f;
#pragma unroll
        for (int i = 0; i < NG; i++) g[i] = 0.f;
        site(L[4 * n4 + lane], g, ob);
#pragma unroll
        for (int i = 0; i < NG; i++) G[i] += (double)g[i];
        F += (double)ob;
    }
#pragma unroll
    for (int i = 0; i < NH; i++) H[i] += (double)h[i];
#pragma unroll
    for (int i = 0; i < NG; i++) out.m[GOFF + i] = G[i];
#pragma unroll
    for (int i = 0; i < NH; i++) out.m[HOFF + i] = H[i];
    out.obj += F;
}

// ----------------------------------------------------------- FP64 passes

// The same sums in FP64 with IEEE division and the library log (the plain
// FP64 form, and the re-evaluation of ill-conditioned or stalled pairs).
template <int S>
__device__ __noinline__ void stream64(const double* __restrict__ L, int64_t len, const PassCoef* K,
                                      int lane, LaneSums& out) {
    constexpr int NG = S == 0 ? 4 : S == 3 ? 4 : S == 4 ? 2 : 3;
    constexpr int NH = S == 0 ? 7 : S == 3 ? 9 : S == 4 ? 3 : 5;
    constexpr int GOFF = S == 0 ? 0 : S == 1 ? 11 : S == 2 ? 19 : S == 3 ? 27 : 40;
    constexpr int HOFF = GOFF + NG;
    const double EPS = 1e-8;
    double k0, k1, k2 = 0.0, k3 = 0.0;
    if (S == 0) { k0 = ld_volatile(&K->a[0]); k1 = ld_volatile(&K->a[1]); k2 = ld_volatile(&K->a[2]); k3 = ld_volatile(&K->a[3]); }
    if (S == 1) { k0 = ld_volatile(&K->b1[0]); k1 = ld_volatile(&K->b1[1]); k2 = ld_volatile(&K->b1[2]); }
    if (S == 2) { k0 = ld_volatile(&K->b2[0]); k1 = ld_volatile(&K->b2[1]); k2 = ld_volatile(&K->b2[2]); }
    if (S == 3) { k0 = ld_volatile(&K->c[0]); k1 = ld_volatile(&K->c[1]); k2 = ld_volatile(&K->c[2]); k3 = ld_volatile(&K->c[3]); }
    if (S == 4) { k0 = ld_volatile(&K->d[0]); k1 = ld_volatile(&K->d[1]); }
    double g[NG], h[NH], F = 0.0;
#pragma unroll
    for (int i = 0; i < NG; i++) g[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NH; i++) h[i] = 0.0;
    auto site = [&](double t) {
        double d;
        if (S == 0) {
            d = fma(t, fma(fma(fma(k3, t, k2), t, k1), t, k0), EPS);
            double r = 1.0 / d;
            double u = r * t;
            double t2 = t * t, t3 = t2 * t, t4 = t2 * t2, t5 = t4 * t, t6 = t3 * t3;
            g[0] += u; g[1] = fma(u, t, g[1]); g[2] = fma(u, t2, g[2]); g[3] = fma(u, t3, g[3]);
            double u2 = u * u;
            h[0] += u2; h[1] = fma(u2, t, h[1]); h[2] = fma(u2, t2, h[2]); h[3] = fma(u2, t3, h[3]);
            h[4] = fma(u2, t4, h[4]); h[5] = fma(u2, t5, h[5]); h[6] = fma(u2, t6, h[6]);
        } else if (S == 1 || S == 2) {
            double w = t * (1.0 - t);
            d = fma(w, fma(fma(k2, t, k1), t, k0), EPS);
            double r = 1.0 / d;
            double v = r * w;
            double t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
            g[0] += v; g[1] = fma(v, t, g[1]); g[2] = fma(v, t2, g[2]);
            double v2 = v * v;
            h[0] += v2; h[1] = fma(v2, t, h[1]); h[2] = fma(v2, t2, h[2]); h[3] = fma(v2, t3, h[3]);
            h[4] = fma(v2, t4, h[4]);
        } else if (S == 3) {
            double ty = 1.0 - t;
            double w = t * ty;
            d = fma(w, fma(w, k3, fma(t, k2, fma(ty, k1, k0))), EPS);
            double r = 1.0 / d;
            double v = r * w;
            g[0] += v; g[1] = fma(v, ty, g[1]); g[2] = fma(v, t, g[2]); g[3] = fma(v, w, g[3]);
            double v2 = v * v;
            h[0] += v2; h[1] = fma(v2, ty, h[1]); h[2] = fma(v2, t, h[2]); h[3] = fma(v2, w, h[3]);
            h[4] = fma(v2, ty * ty, h[4]); h[5] = fma(v2, t * t, h[5]);
            h[6] = fma(v2, w * ty, h[6]); h[7] = fma(v2, w * t, h[7]); h[8] = fma(v2, w * w, h[8]);
        } else {
            double w = t * (1.0 - t);
            d = fma(w, fma(w, k1, k0), EPS);
            double r = 1.0 / d;
            double v = r * w;
            g[0] += v; g[1] = fma(v, w, g[1]);
            double v2 = v * v;
            h[0] += v2; h[1] = fma(v2, w, h[1]); h[2] = fma(v2, w * w, h[2]);
        }
        F += log(d);
    };
    const int64_t n2 = len >> 1;
    const double2* L2 = reinterpret_cast<const double2*>(L);
    const double2 z2 = make_double2(0.0, 0.0);
    int64_t k = lane;
    double2 va = (k < n2) ? L2[k] : z2;
    double2 vb = (k + 32 < n2) ? L2[k + 32] : z2;
    while (k < n2) {
        site(va.x);
        site(va.y);
        va = (k + 64 < n2) ? L2[k + 64] : z2;
        if (k + 32 < n2) {
            site(vb.x);
            site(vb.y);
        }
        vb = (k + 96 < n2) ? L2[k + 96] : z2;
        k += 64;
    }
    if (lane == 0 && (len & 1)) site(L[len - 1]);
#pragma unroll
    for (int i = 0; i < NG; i++) out.m[GOFF + i] = g[i];
#pragma unroll
    for (int i = 0; i < NH; i++) out.m[HOFF + i] = h[i];
    out.obj += F;
}

// ----------------------------------------------------------- reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------- pair SQP

// Pass kinds: the ML passes (FP32 lists with the direct or the difference
// objective; FP64) and the single CLS moment pass (FP32 or FP64 lists).
enum : int { PASS_FP32_DIRECT = 0, PASS_FP32_DIFF = 1, PASS_FP64 = 2, PASS_CLS = 3, PASS_CLS64 = 4 };

struct PairEval {
    double f;       // objective at the evaluated point
    double g[9];    // gradient (warp-uniform)
    double Hr[9];   // this lane's row of the Hessian (lanes 0..8)
};

__constant__ int kEA[9] = {1, 2, 2, 3, 2, 3, 2, 3, 4};      // t-power of each entry in shape A
__constant__ int kPosB1[9] = {-1, -1, 0, 1, -1, -1, -1, 2, 3};
__constant__ int kPosB2[9] = {-1, -1, -1, -1, 0, 1, -1, 2, 3};
__constant__ int kPosC[9] = {-1, 0, -1, 1, -1, 2, -1, -1, 3};
__constant__ int kPosD[9] = {-1, -1, -1, -1, -1, -1, 0, 1, 2};
__constant__ int kHC[4][4] = {{0, 1, 2, 3}, {1, 4, 3, 6}, {2, 3, 5, 7}, {3, 6, 7, 8}};

// Row r of S = sum L r and T = sum L L' r^2 from the 45 moment totals (shared
// memory), adding the shapes' contributions in the order A, B1, B2, C, D.
__device__ inline void rebuild_row(const double* mom, int r, double& S, double* T) {
    const int cb[4] = {1, 2, 1, 2};
    const int pb[4] = {0, 1, 1, 2};
    const int i1[4] = {2, 3, 7, 8};
    const int i2[4] = {4, 5, 7, 8};
    const int ic[4] = {1, 3, 5, 8};
    const int id[3] = {6, 7, 8};
    const double cd[3] = {2.0, 1.0, 4.0};
    const int pd[3] = {0, 0, 1};
    const int er = kEA[r];
    S = mom[er - 1];
#pragma unroll
    for (int j = 0; j < 9; j++) {
        const int ej = (j == 0) ? 1 : (j == 8) ? 4 : (j == 3 || j == 5 || j == 7) ? 3 : 2;
        T[j] = mom[4 + er + ej - 2];
    }
    const int a1 = kPosB1[r], a2 = kPosB2[r], ac = kPosC[r], ad = kPosD[r];
    if (a1 >= 0) S += (double)cb[a1] * mom[11 + pb[a1]];
    if (a2 >= 0) S += (double)cb[a2] * mom[19 + pb[a2]];
    if (ac >= 0) S += mom[27 + ac];
    if (ad >= 0) S += (ad == 0 ? 2.0 : ad == 1 ? 1.0 : 4.0) * mom[40 + (ad == 2 ? 1 : 0)];
#pragma unroll
    for (int b = 0; b < 4; b++) {
        if (a1 >= 0) T[i1[b]] += (double)(cb[a1] * cb[b]) * mom[14 + pb[a1] + pb[b]];
        if (a2 >= 0) T[i2[b]] += (double)(cb[a2] * cb[b]) * mom[22 + pb[a2] + pb[b]];
    }
    if (ac >= 0) {
#pragma unroll
        for (int b = 0; b < 4; b++) T[ic[b]] += mom[31 + kHC[ac][b]];
    }
    if (ad >= 0) {
        const double ca = (ad == 0 ? 2.0 : ad == 1 ? 1.0 : 4.0);
        const int pa = (ad == 2 ? 1 : 0);
#pragma unroll
        for (int b = 0; b < 3; b++) T[id[b]] += ca * cd[b] * mom[42 + pa + pd[b]];
    }
}

// Evaluates f, g, H at x from the pair's lists (FP32 lists for the FP32
// kinds, FP64 lists for PASS_FP64).  For PASS_FP32_DIFF,
// f = f_base - (sum log(d/d_base))/n with x_base the accepted point.
__device__ inline void evaluate(const PairLists& pl, const void* lists, int kind, const double* x,
                                const double* x_base, double f_base, int lane, char* wsm,
                                PairEval& ev, unsigned long long& cyc_stream) {
    void* kbuf = wsm + WARP_SMEM_BUF;
    double* mom_s = reinterpret_cast<double*>(wsm);   // NMOM + 1 totals (sort buffer is free)
    PassCoef k;
    make_coef(x, k);
    __syncwarp();
    if (kind == PASS_FP64) {
        if (lane == 0) *reinterpret_cast<PassCoef*>(kbuf) = k;
    } else if (lane == 0) {
        Coef32 c;
        for (int i = 0; i < 4; i++) { c.a[i] = split(k.a[i]); c.c[i] = split(k.c[i]); }
        for (int i = 0; i < 3; i++) { c.b1[i] = split(k.b1[i]); c.b2[i] = split(k.b2[i]); }
        for (int i = 0; i < 2; i++) c.d[i] = split(k.d[i]);
        double s[9];
        for (int i = 0; i < 9; i++) s[i] = x[i] - x_base[i];
        PassCoef ks;
        make_coef(s, ks);
        for (int i = 0; i < 4; i++) { c.sa[i] = (float)ks.a[i]; c.sc[i] = (float)ks.c[i]; }
        for (int i = 0; i < 3; i++) { c.sb1[i] = (float)ks.b1[i]; c.sb2[i] = (float)ks.b2[i]; }
        for (int i = 0; i < 2; i++) c.sd[i] = (float)ks.d[i];
        *reinterpret_cast<Coef32*>(kbuf) = c;
    }
    __syncwarp();
    LaneSums ls;
    ls.obj = 0.0;
    const long long ts0 = clock64();
    if (kind == PASS_FP64) {
        const double* L = static_cast<const double*>(lists);
        const PassCoef* K = reinterpret_cast<const PassCoef*>(kbuf);
        stream64<0>(L + pl.start[0], pl.cnt[0], K, lane, ls);
        stream64<1>(L + pl.start[1], pl.cnt[1], K, lane, ls);
        stream64<2>(L + pl.start[2], pl.cnt[2], K, lane, ls);
        stream64<3>(L + pl.start[3], pl.cnt[3], K, lane, ls);
        stream64<4>(L + pl.start[4], pl.cnt[4], K, lane, ls);
    } else {
        const float* L = static_cast<const float*>(lists);
        const Coef32* K = reinterpret_cast<const Coef32*>(kbuf);
        const bool diff = (kind == PASS_FP32_DIFF);
        stream32<0>(L + pl.start[0], pl.cnt[0], K, diff, lane, ls);
        stream32<1>(L + pl.start[1], pl.cnt[1], K, diff, lane, ls);
        stream32<2>(L + pl.start[2], pl.cnt[2], K, diff, lane, ls);
        stream32<3>(L + pl.start[3], pl.cnt[3], K, diff, lane, ls);
        stream32<4>(L + pl.start[4], pl.cnt[4], K, diff, lane, ls);
    }
    cyc_stream += clock64() - ts0;
    for (int i = 0; i < NMOM; i++) {
        const double v = warp_sum(ls.m[i]);
        if (lane == 0) mom_s[i] = v;
    }
    const double obj = warp_sum(ls.obj);
    __syncwarp();
    const double n = (double)pl.n;
    double S = 0.0;
#pragma unroll
    for (int j = 0; j < 9; j++) ev.Hr[j] = 0.0;
    if (lane < 9) {
        rebuild_row(mom_s, lane, S, ev.Hr);
#pragma unroll
        for (int j = 0; j < 9; j++) ev.Hr[j] = ev.Hr[j] / n;
    }
    gather9(-S / n, ev.g);
    __syncwarp();
    if (kind == PASS_FP64) {
        ev.f = -obj / n;
    } else if (kind == PASS_FP32_DIRECT) {
        ev.f = -(obj * 0.69314718055994530942) / n;
    } else {
        ev.f = f_base - obj / n;
    }
}

constexpr double COND_RECHECK = 1e4;   // FP32 condition estimates above this are redone in FP64
// |alpha g.p| under which the objective change is summed directly.  The
// direct FP32 objective (one lg2 per four sites, rounding ~3e-7 in log2 units
// per call, independent across calls) is off by ~3e-10 at n = 1e5 sites, and
// the Armijo test's margin is about |alpha g.p| / 2: at 1e-7 that margin is
// ~70 times the error of the difference f_new - f_old.
constexpr double DIFF_BELOW = 1e-7;

struct PairResult {
    unsigned long long cyc_pass;    // clocks spent in site passes
    unsigned long long cyc_stream;  // of which inside the shape streams
    unsigned long long cyc_solve;   // clocks spent in the 9x9 solver steps
    double x[9];
    double f;
    uint64_t iters;
    double cond;
    int fp64_passes;
    int gh_passes;
    int obj_passes;
    int diff_passes;
    bool escalated;
};

// Executed site arithmetic per pass and shape (A, B1, B2, C, D), counting an
// FMA as 2 and a MUFU op as 1, read off Shape32 and stream64.  The wave engine
// (hi coefficients, one lg2 per four sites) is counted per four sites, with the
// extra of the log(d_new/d_old) objective beside it; the single-kernel engine
// (hi + lo polynomial, one lg2 per site) and FP64 passes per site.
__host__ __device__ constexpr int flops4_fp32_hi(int s) {
    return s == 0 ? 141 : s == 1 ? 113 : s == 2 ? 113 : s == 3 ? 165 : 77;
}
__host__ __device__ constexpr int flops4_diff_extra(int s) {
    return s == 0 ? 48 : s == 1 ? 40 : s == 2 ? 40 : s == 3 ? 52 : 32;
}
__host__ __device__ constexpr int flops_fp32_lo(int s) {
    return s == 0 ? 43 : s == 1 ? 34 : s == 2 ? 34 : s == 3 ? 49 : 23;
}
__host__ __device__ constexpr int flops_fp64(int s) {
    return s == 0 ? 50 : s == 1 ? 39 : s == 2 ? 39 : s == 3 ? 55 : 27;
}
__host__ __device__ constexpr int flops_diff_extra(int s) {
    return s == 0 ? 18 : s == 1 ? 16 : s == 2 ? 16 : s == 3 ? 19 : 14;
}

// Condition estimate from the row-distributed Hessian (once per pair).
template <class G>
__device__ inline double condition_rows(const G& grp, const double* x, const double* g, const double* Hr,
                                        double tol) {
    double H[81];
#pragma unroll
    for (int i = 0; i < 9; i++)
#pragma unroll
        for (int j = 0; j < 9; j++) H[i * 9 + j] = grp.bcast(Hr[j], i);
    return condition_estimate(x, g, H, tol);
}
__device__ inline double condition_rows(const double* x, const double* g, const double* Hr, double tol) {
    return condition_rows(WarpGrp{FULL_MASK}, x, g, Hr, tol);
}

// SQP of one pair (src/sqp.rs:49-93) over its sorted lists.  The FP32 lists
// are replaced by FP64 lists when the pair escalates.
__device__ inline void solve_pair(const CohortDev& co, int64_t px, int64_t py, const PairLists& pl,
                                  void* lists, bool self_pair, int precision, const Tune& tu,
                                  int lane, char* wsm, PairResult& res) {
    double x[9];
#pragma unroll
    for (int i = 0; i < 9; i++) x[i] = self_pair ? 0.0 : 1.0 / 9.0;
    if (self_pair) { x[0] = 0.5; x[6] = 0.5; }
    normalise9(x);
    bool fp64 = (precision == 1);
    res.fp64_passes = 0;
    res.gh_passes = 0;
    res.obj_passes = 0;
    res.diff_passes = 0;
    res.escalated = false;
    res.cyc_pass = 0;
    res.cyc_solve = 0;
    res.cyc_stream = 0;
    PairEval ev;
    const long long t_0 = clock64();
    evaluate(pl, lists, fp64 ? PASS_FP64 : PASS_FP32_DIRECT, x, x, 0.0, lane, wsm, ev, res.cyc_stream);
    res.cyc_pass += clock64() - t_0;
    res.obj_passes++;
    res.gh_passes++;
    if (fp64) res.fp64_passes++;
    double f = ev.f;
    double g[9], Hr[9];
#pragma unroll
    for (int i = 0; i < 9; i++) { g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
    int near_count = 0;
    for (uint64_t it = 0; it < tu.sqp_max_iter; it++) {
        double resid;
        bool conv = kkt_ok(x, g, tu.sqp_conv_tol, &resid);
        if (!fp64 && (conv || resid < 1e-6)) {
            if (!conv) near_count++;
            double cond = conv ? condition_rows(x, g, Hr, tu.sqp_conv_tol) : 0.0;
            bool recheck = conv ? !(cond <= COND_RECHECK) : (near_count >= 3);
            if (recheck) {
                // FP64 re-evaluation at the same point; the pair stays FP64 from here.
                scatter_shapes<double>(co, px, py, lane, pl, static_cast<double*>(lists), wsm);
                const long long ta = clock64();
                evaluate(pl, lists, PASS_FP64, x, x, f, lane, wsm, ev, res.cyc_stream);
                res.cyc_pass += clock64() - ta;
                res.fp64_passes++;
                res.gh_passes++;
                res.obj_passes++;
                fp64 = true;
                res.escalated = true;
                f = ev.f;
#pragma unroll
                for (int i = 0; i < 9; i++) { g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
                conv = kkt_ok(x, g, tu.sqp_conv_tol, &resid);
            } else if (conv) {
#pragma unroll
                for (int i = 0; i < 9; i++) res.x[i] = x[i];
                res.f = f;
                res.iters = it;
                res.cond = cond;
                res.cyc_solve = (clock64() - t_0) - res.cyc_pass;
                return;
            }
        }
        if (conv) {
#pragma unroll
            for (int i = 0; i < 9; i++) res.x[i] = x[i];
            res.f = f;
            res.iters = it;
            res.cond = condition_rows(x, g, Hr, tu.sqp_conv_tol);
            res.cyc_solve = (clock64() - t_0) - res.cyc_pass;
            return;
        }
        // QP step: c = g - H x
        double cr = 0.0;
        if (lane < 9) cr = pick9(g, lane) - dot_fma(9, Hr, x);
        double c[9], y[9], p[9];
        gather9(cr, c);
        qp_simplex_rows(WarpGrp{FULL_MASK}, Hr, c, x, tu, lane, y);
#pragma unroll
        for (int i = 0; i < 9; i++) p[i] = y[i] - x[i];
        const double gp = dot_fma(9, g, p);
        const double tt = tu.bls_sufficient_decrease * gp;
        double alpha = 1.0;
        double xn[9];
        for (int bls = 0;;) {
#pragma unroll
            for (int i = 0; i < 9; i++) xn[i] = x[i] + alpha * p[i];
            normalise9(xn);
            const int kind = fp64 ? PASS_FP64
                                  : (fabs(alpha * gp) < DIFF_BELOW ? PASS_FP32_DIFF : PASS_FP32_DIRECT);
            const long long ta = clock64();
            evaluate(pl, lists, kind, xn, x, f, lane, wsm, ev, res.cyc_stream);
            res.cyc_pass += clock64() - ta;
            res.obj_passes++;
            res.gh_passes++;
            if (kind == PASS_FP64) res.fp64_passes++;
            if (kind == PASS_FP32_DIFF) res.diff_passes++;
            const bool accept = ev.f <= f + alpha * tt;
            bls++;
            if (accept || bls == tu.bls_max_iter) break;
            alpha *= tu.bls_step_size_reduce;
        }
#pragma unroll
        for (int i = 0; i < 9; i++) { x[i] = xn[i]; g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
        f = ev.f;
    }
#pragma unroll
    for (int i = 0; i < 9; i++) res.x[i] = x[i];
    res.f = f;
    res.iters = tu.sqp_max_iter;
    res.cond = CUDART_NAN;
    res.cyc_solve = (clock64() - t_0) - res.cyc_pass;
}

}  // namespace kg
