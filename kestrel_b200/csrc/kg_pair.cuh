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
// Precision (KG_PREC_FP32C): per-site terms in FP32 with MUFU rcp/lg2 plus a
// Newton step, the pair's coefficients split hi+lo so the evaluation point is
// the exact FP64 iterate, FP32 partial sums promoted to FP64 per segment, and
// near convergence the objective change is summed directly as
// log(d_new/d_old) = -log1p(-delta/d_new) so the Armijo test (src/sqp.rs:294)
// keeps its resolution.  The 9x9 QP, LDL^T, KKT and condition estimate are
// FP64.  Pairs whose condition estimate is large, or whose FP32 KKT residual
// stalls, are re-evaluated with FP64 passes.
#pragma once

#include <cstdint>
#include <math_constants.h>

#include "kestrel_gpu.h"
#include "kg_solver.cuh"

namespace kg {

constexpr int SEG_SITES = 2048;             // sites per segment
constexpr int SEG_WORDS = SEG_SITES / 32;   // 32-site plane words per segment
constexpr int SEG_HDR = 8;                  // u16 header entries per segment

enum : int { COHORT_TRIANGLE = 0, COHORT_RECT = 1 };

// Device-side description of one cohort (or one serving request).
struct CohortDev {
    const uint2* planes_x;   // [rows_x][plane_stride] {lo, hi} bit planes of 32 sites
    const uint2* planes_y;   // [rows_y][plane_stride] (== planes_x for a triangle)
    int64_t plane_stride;    // words per row (multiple of SEG_WORDS)
    const float* p32;        // REF frequency per kept site, padded
    const double* p64;
    const double* q64;
    int32_t n_sites;         // kept (segregating) sites
    int32_t n_segments;
    int32_t kind;            // COHORT_TRIANGLE or COHORT_RECT
    int32_t pad;
    int64_t n_x;             // triangle: num_samples; rect: query rows
    int64_t n_y;             // rect: panel rows
    int64_t pair_begin;      // first global work index
    int64_t n_pairs;
    kg_output* out;          // rows in the reference's order
};

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
};

struct PairLaunch {
    const CohortDev* cohorts;
    int n_cohorts;
    int precision;               // 0 FP32C, 1 FP64
    int64_t total_pairs;
    unsigned long long* queue;   // next work index
    uint16_t* scratch;           // per warp: [n_seg_max * SEG_SITES] entries
    uint16_t* headers;           // per warp: [n_seg_max * SEG_HDR]
    int64_t scratch_stride;      // entries per warp
    int64_t header_stride;       // header u16 per warp
    Tune tune;
    RunCounters* counters;
};

// ------------------------------------------------------------ FP32 helpers

__device__ __forceinline__ float rcp_nr(float d) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
    float e = fmaf(-d, r, 1.0f);
    return fmaf(r, e, r);
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

// Moment accumulators (FP64 totals), in the order used by the rebuild:
//  0..3  GA  sum r t^k, k=1..4          4..10 HA  sum r^2 t^k, k=2..8
// 11..13 GB1 sum r w t^k, k=0..2        14..18 HB1 sum r^2 w^2 t^k, k=0..4
// 19..21 GB2                            22..26 HB2
// 27..30 GC  sum r w {1,ty,tx,w}        31..39 HC sum r^2 w^2 {1,ty,tx,w,ty^2,tx^2,w ty,w tx,w^2}
// 40..41 GD  sum r w {1,w}              42..44 HD  sum r^2 w^2 {1,w,w^2}
constexpr int NMOM = 45;

struct PassOut {
    double mom[NMOM];
    double obj;      // sum of lg2(d) [FP32 direct], log(d) [FP64], or log(d_new/d_old) [diff]
};

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

// Builds the per-segment shape lists of pair (x, y) in this warp's scratch.
// Entry = site-in-segment (11 bits) | sel << 15, where sel picks t = q.
// Header per segment: {startB1, startB2, startC, startD, total}.
// Returns the number of jointly observed segregating sites.
__device__ inline int64_t sort_pair(const CohortDev& co, int64_t x, int64_t y, uint16_t* ent,
                                    uint16_t* hdr, uint16_t* buf, int lane, int64_t* shape_n) {
    const uint2* px = co.planes_x + x * co.plane_stride;
    const uint2* py = co.planes_y + y * co.plane_stride;
    int64_t n = 0;
    for (int s = 0; s < 5; s++) shape_n[s] = 0;
    for (int seg = 0; seg < co.n_segments; seg++) {
        uint32_t m[2][5], sel[2];
        unsigned cnt[5] = {0, 0, 0, 0, 0};
#pragma unroll
        for (int h = 0; h < 2; h++) {
            uint2 X = px[seg * SEG_WORDS + h * 32 + lane];
            uint2 Y = py[seg * SEG_WORDS + h * 32 + lane];
            uint32_t xhom = ~X.x, xhet = X.x & ~X.y;
            uint32_t yhom = ~Y.x, yhet = Y.x & ~Y.y;
            uint32_t same = ~(X.y ^ Y.y);
            m[h][0] = xhom & yhom & same;   // A
            m[h][1] = xhom & yhet;          // B1
            m[h][2] = xhet & yhom;          // B2
            m[h][3] = xhom & yhom & ~same;  // C
            m[h][4] = xhet & yhet;          // D
            sel[h] = (X.y & ~m[h][2]) | (Y.y & m[h][2]);
#pragma unroll
            for (int s = 0; s < 5; s++) cnt[s] += __popc(m[h][s]);
        }
        // warp-exclusive scan of the five counts packed in 12-bit fields
        unsigned long long v = 0;
#pragma unroll
        for (int s = 0; s < 5; s++) v |= (unsigned long long)cnt[s] << (12 * s);
        unsigned long long inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        unsigned long long tot = __shfl_sync(0xffffffffu, inc, 31);
        unsigned long long exc = inc - v;
        unsigned start[6];
        start[0] = 0;
#pragma unroll
        for (int s = 0; s < 5; s++) start[s + 1] = start[s] + (unsigned)((tot >> (12 * s)) & 0xFFF);
        unsigned pos[5];
#pragma unroll
        for (int s = 0; s < 5; s++) pos[s] = start[s] + (unsigned)((exc >> (12 * s)) & 0xFFF);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            unsigned base = (unsigned)((h * 32 + lane) * 32);
#pragma unroll
            for (int s = 0; s < 5; s++) {
                uint32_t mm = m[h][s];
                while (mm) {
                    int i = __ffs(mm) - 1;
                    mm &= mm - 1;
                    unsigned e = (base + i) | (((sel[h] >> i) & 1u) << 15);
                    buf[pos[s]++] = (uint16_t)e;
                }
            }
        }
        __syncwarp();
        // copy the segment's entries out (4 KB) with 16-byte stores
        const uint4* src = reinterpret_cast<const uint4*>(buf);
        uint4* dst = reinterpret_cast<uint4*>(ent + (int64_t)seg * SEG_SITES);
        unsigned total = start[5];
        unsigned nvec = (total + 7) / 8;
        for (unsigned k = lane; k < nvec; k += 32) dst[k] = src[k];
        if (lane == 0) {
            uint4 h4;
            h4.x = start[1] | (start[2] << 16);
            h4.y = start[3] | (start[4] << 16);
            h4.z = total;
            h4.w = 0;
            *reinterpret_cast<uint4*>(hdr + (int64_t)seg * SEG_HDR) = h4;
        }
        __syncwarp();
        n += total;
#pragma unroll
        for (int s = 0; s < 5; s++) shape_n[s] += start[s + 1] - start[s];
    }
    return n;
}

// ----------------------------------------------------------- FP32 passes

enum : int { OBJ_DIRECT = 0, OBJ_DIFF = 1 };

// Warp-uniform pass coefficients, kept in shared memory and re-read at the top
// of each shape loop so only the current shape's values occupy registers.
struct Coef32 {
    HiLo a[4], b1[3], b2[3], c[4], d[2];
    float sa[4], sb1[3], sb2[3], sc[4], sd[2];  // step coefficients (OBJ_DIFF)
};

// Shared-memory words per warp: the FP64 accumulators (NACC per lane, lane-
// interleaved) overlay the 2048-entry sort buffer; the coefficients follow.
constexpr int NACC = NMOM + 1;  // moments + objective
constexpr int WARP_SMEM_ACC = NACC * 32 * 8;
constexpr int WARP_SMEM_COEF = 512;
constexpr int WARP_SMEM = WARP_SMEM_ACC + WARP_SMEM_COEF;
static_assert(WARP_SMEM_ACC >= SEG_SITES * 2, "sort buffer must fit under the accumulators");
static_assert(sizeof(Coef32) <= WARP_SMEM_COEF, "coefficients must fit");

// acc points at this lane's first accumulator (stride 32 doubles).
__device__ __forceinline__ void acc_add(double* acc, int i, double v) { acc[i * 32] += v; }

template <class T>
__device__ __forceinline__ T ld_volatile(const T* p) { return *reinterpret_cast<const volatile T*>(p); }

__device__ __forceinline__ HiLo ldk(const HiLo* p) {
    HiLo r;
    r.h = ld_volatile(&p->h);
    r.l = ld_volatile(&p->l);
    return r;
}

// Sums over one pair's lists at the FP32 evaluation point into this lane's
// shared-memory accumulators.
template <int OBJ>
__device__ __noinline__ void pass_fp32(const CohortDev& co, const uint16_t* ent, const uint16_t* hdr,
                                       const Coef32* K, double* acc, int lane) {
    const float EPS = 1e-8f;
    for (int seg = 0; seg < co.n_segments; seg++) {
        uint4 h4 = *reinterpret_cast<const uint4*>(hdr + (int64_t)seg * SEG_HDR);
        const int sB1 = h4.x & 0xFFFF, sB2 = h4.x >> 16, sC = h4.y & 0xFFFF, sD = h4.y >> 16;
        const int tot = h4.z;
        const uint16_t* E = ent + (int64_t)seg * SEG_SITES;
        const float* P = co.p32 + (int64_t)seg * SEG_SITES;
        // ---- shape A
        {
            const HiLo a0 = ldk(&K->a[0]), a1 = ldk(&K->a[1]), a2 = ldk(&K->a[2]), a3 = ldk(&K->a[3]);
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
            if (OBJ == OBJ_DIFF) {
                s0 = ld_volatile(&K->sa[0]); s1 = ld_volatile(&K->sa[1]);
                s2 = ld_volatile(&K->sa[2]); s3 = ld_volatile(&K->sa[3]);
            }
            float g0 = 0, g1 = 0, g2 = 0, g3 = 0, h0 = 0, h1 = 0, h2 = 0, h3 = 0, h4_ = 0, h5 = 0, h6 = 0, ob = 0;
#pragma unroll 2
            for (int j = lane; j < sB1; j += 32) {
                unsigned e = E[j];
                float p = P[e & 0x7FF];
                float t = (e >> 15) ? 1.0f - p : p;
                float t2 = t * t, t3 = t2 * t, t4 = t2 * t2, t5 = t4 * t, t6 = t3 * t3;
                float ph = fmaf(fmaf(fmaf(a3.h, t, a2.h), t, a1.h), t, a0.h);
                float pl = fmaf(fmaf(fmaf(a3.l, t, a2.l), t, a1.l), t, a0.l);
                float d = fmaf(t, ph + pl, EPS);
                float r = rcp_nr(d);
                float u = r * t;
                g0 += u; g1 = fmaf(u, t, g1); g2 = fmaf(u, t2, g2); g3 = fmaf(u, t3, g3);
                float u2 = u * u;
                h0 += u2; h1 = fmaf(u2, t, h1); h2 = fmaf(u2, t2, h2); h3 = fmaf(u2, t3, h3);
                h4_ = fmaf(u2, t4, h4_); h5 = fmaf(u2, t5, h5); h6 = fmaf(u2, t6, h6);
                if (OBJ == OBJ_DIRECT) {
                    ob += lg2_approx(d);
                } else {
                    float dl = t * fmaf(fmaf(fmaf(s3, t, s2), t, s1), t, s0);
                    ob += neg_log1m(dl * r);
                }
            }
            acc_add(acc, 0, g0); acc_add(acc, 1, g1); acc_add(acc, 2, g2); acc_add(acc, 3, g3);
            acc_add(acc, 4, h0); acc_add(acc, 5, h1); acc_add(acc, 6, h2); acc_add(acc, 7, h3);
            acc_add(acc, 8, h4_); acc_add(acc, 9, h5); acc_add(acc, 10, h6);
            acc_add(acc, NMOM, ob);
        }
        // ---- shapes B1 and B2 (same form, different coefficients and moments)
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const HiLo* kb = b ? K->b2 : K->b1;
            const float* sbp = b ? K->sb2 : K->sb1;
            const HiLo k0 = ldk(&kb[0]), k1 = ldk(&kb[1]), k2 = ldk(&kb[2]);
            float s0 = 0.f, s1 = 0.f, s2 = 0.f;
            if (OBJ == OBJ_DIFF) { s0 = ld_volatile(&sbp[0]); s1 = ld_volatile(&sbp[1]); s2 = ld_volatile(&sbp[2]); }
            const int lo = b ? sB2 : sB1, hi = b ? sC : sB2;
            float g0 = 0, g1 = 0, g2 = 0, h0 = 0, h1 = 0, h2 = 0, h3 = 0, h4_ = 0, ob = 0;
#pragma unroll 2
            for (int j = lo + lane; j < hi; j += 32) {
                unsigned e = E[j];
                float p = P[e & 0x7FF];
                float q = 1.0f - p;
                float t = (e >> 15) ? q : p;
                float w = p * q;
                float t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
                float ph = fmaf(fmaf(k2.h, t, k1.h), t, k0.h);
                float pl = fmaf(fmaf(k2.l, t, k1.l), t, k0.l);
                float d = fmaf(w, ph + pl, EPS);
                float r = rcp_nr(d);
                float v = r * w;
                g0 += v; g1 = fmaf(v, t, g1); g2 = fmaf(v, t2, g2);
                float v2 = v * v;
                h0 += v2; h1 = fmaf(v2, t, h1); h2 = fmaf(v2, t2, h2); h3 = fmaf(v2, t3, h3);
                h4_ = fmaf(v2, t4, h4_);
                if (OBJ == OBJ_DIRECT) {
                    ob += lg2_approx(d);
                } else {
                    float dl = w * fmaf(fmaf(s2, t, s1), t, s0);
                    ob += neg_log1m(dl * r);
                }
            }
            const int gb = b ? 19 : 11, hb = b ? 22 : 14;
            acc_add(acc, gb + 0, g0); acc_add(acc, gb + 1, g1); acc_add(acc, gb + 2, g2);
            acc_add(acc, hb + 0, h0); acc_add(acc, hb + 1, h1); acc_add(acc, hb + 2, h2);
            acc_add(acc, hb + 3, h3); acc_add(acc, hb + 4, h4_);
            acc_add(acc, NMOM, ob);
        }
        // ---- shape C
        {
            const HiLo c0 = ldk(&K->c[0]), c1 = ldk(&K->c[1]), c2 = ldk(&K->c[2]), c3 = ldk(&K->c[3]);
            float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
            if (OBJ == OBJ_DIFF) {
                s0 = ld_volatile(&K->sc[0]); s1 = ld_volatile(&K->sc[1]);
                s2 = ld_volatile(&K->sc[2]); s3 = ld_volatile(&K->sc[3]);
            }
            float g0 = 0, g1 = 0, g2 = 0, g3 = 0, ob = 0;
            float h[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int j = sC + lane; j < sD; j += 32) {
                unsigned e = E[j];
                float p = P[e & 0x7FF];
                float q = 1.0f - p;
                bool s = (e >> 15) != 0;
                float tx = s ? q : p, ty = s ? p : q;
                float w = p * q;
                float ph = fmaf(w, c3.h, fmaf(tx, c2.h, fmaf(ty, c1.h, c0.h)));
                float pl = fmaf(w, c3.l, fmaf(tx, c2.l, fmaf(ty, c1.l, c0.l)));
                float d = fmaf(w, ph + pl, EPS);
                float r = rcp_nr(d);
                float v = r * w;
                g0 += v; g1 = fmaf(v, ty, g1); g2 = fmaf(v, tx, g2); g3 = fmaf(v, w, g3);
                float v2 = v * v;
                h[0] += v2; h[1] = fmaf(v2, ty, h[1]); h[2] = fmaf(v2, tx, h[2]); h[3] = fmaf(v2, w, h[3]);
                h[4] = fmaf(v2, ty * ty, h[4]); h[5] = fmaf(v2, tx * tx, h[5]);
                h[6] = fmaf(v2, w * ty, h[6]); h[7] = fmaf(v2, w * tx, h[7]); h[8] = fmaf(v2, w * w, h[8]);
                if (OBJ == OBJ_DIRECT) {
                    ob += lg2_approx(d);
                } else {
                    float dl = w * fmaf(w, s3, fmaf(tx, s2, fmaf(ty, s1, s0)));
                    ob += neg_log1m(dl * r);
                }
            }
            acc_add(acc, 27, g0); acc_add(acc, 28, g1); acc_add(acc, 29, g2); acc_add(acc, 30, g3);
#pragma unroll
            for (int i = 0; i < 9; i++) acc_add(acc, 31 + i, h[i]);
            acc_add(acc, NMOM, ob);
        }
        // ---- shape D
        {
            const HiLo d0 = ldk(&K->d[0]), d1 = ldk(&K->d[1]);
            float s0 = 0.f, s1 = 0.f;
            if (OBJ == OBJ_DIFF) { s0 = ld_volatile(&K->sd[0]); s1 = ld_volatile(&K->sd[1]); }
            float g0 = 0, g1 = 0, h0 = 0, h1 = 0, h2 = 0, ob = 0;
            for (int j = sD + lane; j < tot; j += 32) {
                unsigned e = E[j];
                float p = P[e & 0x7FF];
                float w = p * (1.0f - p);
                float ph = fmaf(w, d1.h, d0.h);
                float pl = fmaf(w, d1.l, d0.l);
                float d = fmaf(w, ph + pl, EPS);
                float r = rcp_nr(d);
                float v = r * w;
                g0 += v; g1 = fmaf(v, w, g1);
                float v2 = v * v;
                h0 += v2; h1 = fmaf(v2, w, h1); h2 = fmaf(v2, w * w, h2);
                if (OBJ == OBJ_DIRECT) {
                    ob += lg2_approx(d);
                } else {
                    float dl = w * fmaf(w, s1, s0);
                    ob += neg_log1m(dl * r);
                }
            }
            acc_add(acc, 40, g0); acc_add(acc, 41, g1);
            acc_add(acc, 42, h0); acc_add(acc, 43, h1); acc_add(acc, 44, h2);
            acc_add(acc, NMOM, ob);
        }
    }
}

// ----------------------------------------------------------- FP64 passes

// The same sums in FP64 with IEEE division and the library log (the plain
// FP64 form); per-shape partials are flushed to the shared accumulators.
__device__ __noinline__ void pass_fp64(const CohortDev& co, const uint16_t* ent, const uint16_t* hdr,
                                       const PassCoef* Kp, double* acc, int lane) {
    const double EPS = 1e-8;
    for (int seg = 0; seg < co.n_segments; seg++) {
        uint4 h4 = *reinterpret_cast<const uint4*>(hdr + (int64_t)seg * SEG_HDR);
        const int sB1 = h4.x & 0xFFFF, sB2 = h4.x >> 16, sC = h4.y & 0xFFFF, sD = h4.y >> 16;
        const int tot = h4.z;
        const uint16_t* E = ent + (int64_t)seg * SEG_SITES;
        const double* P = co.p64 + (int64_t)seg * SEG_SITES;
        const double* Q = co.q64 + (int64_t)seg * SEG_SITES;
        {
            const double a0 = ld_volatile(&Kp->a[0]), a1 = ld_volatile(&Kp->a[1]);
            const double a2 = ld_volatile(&Kp->a[2]), a3 = ld_volatile(&Kp->a[3]);
            double m[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            double ob = 0.0;
            for (int j = lane; j < sB1; j += 32) {
                unsigned e = E[j];
                double t = (e >> 15) ? Q[e & 0x7FF] : P[e & 0x7FF];
                double t2 = t * t, t3 = t2 * t, t4 = t2 * t2, t5 = t4 * t, t6 = t3 * t3;
                double d = fma(t, fma(fma(fma(a3, t, a2), t, a1), t, a0), EPS);
                double r = 1.0 / d;
                double u = r * t;
                m[0] += u; m[1] = fma(u, t, m[1]); m[2] = fma(u, t2, m[2]); m[3] = fma(u, t3, m[3]);
                double u2 = u * u;
                m[4] += u2; m[5] = fma(u2, t, m[5]); m[6] = fma(u2, t2, m[6]); m[7] = fma(u2, t3, m[7]);
                m[8] = fma(u2, t4, m[8]); m[9] = fma(u2, t5, m[9]); m[10] = fma(u2, t6, m[10]);
                ob += log(d);
            }
#pragma unroll
            for (int i = 0; i < 11; i++) acc_add(acc, i, m[i]);
            acc_add(acc, NMOM, ob);
        }
#pragma unroll
        for (int b = 0; b < 2; b++) {
            const double* kb = b ? Kp->b2 : Kp->b1;
            const double k0 = ld_volatile(&kb[0]), k1 = ld_volatile(&kb[1]), k2 = ld_volatile(&kb[2]);
            const int lo = b ? sB2 : sB1, hi = b ? sC : sB2;
            double m[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            double ob = 0.0;
            for (int j = lo + lane; j < hi; j += 32) {
                unsigned e = E[j];
                double p = P[e & 0x7FF], q = Q[e & 0x7FF];
                double t = (e >> 15) ? q : p;
                double w = p * q;
                double t2 = t * t, t3 = t2 * t, t4 = t2 * t2;
                double d = fma(w, fma(fma(k2, t, k1), t, k0), EPS);
                double r = 1.0 / d;
                double v = r * w;
                m[0] += v; m[1] = fma(v, t, m[1]); m[2] = fma(v, t2, m[2]);
                double v2 = v * v;
                m[3] += v2; m[4] = fma(v2, t, m[4]); m[5] = fma(v2, t2, m[5]); m[6] = fma(v2, t3, m[6]);
                m[7] = fma(v2, t4, m[7]);
                ob += log(d);
            }
            const int gb = b ? 19 : 11, hb = b ? 22 : 14;
#pragma unroll
            for (int i = 0; i < 3; i++) acc_add(acc, gb + i, m[i]);
#pragma unroll
            for (int i = 0; i < 5; i++) acc_add(acc, hb + i, m[3 + i]);
            acc_add(acc, NMOM, ob);
        }
        {
            const double c0 = ld_volatile(&Kp->c[0]), c1 = ld_volatile(&Kp->c[1]);
            const double c2 = ld_volatile(&Kp->c[2]), c3 = ld_volatile(&Kp->c[3]);
            double m[13] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            double ob = 0.0;
            for (int j = sC + lane; j < sD; j += 32) {
                unsigned e = E[j];
                double p = P[e & 0x7FF], q = Q[e & 0x7FF];
                bool s = (e >> 15) != 0;
                double tx = s ? q : p, ty = s ? p : q;
                double w = p * q;
                double d = fma(w, fma(w, c3, fma(tx, c2, fma(ty, c1, c0))), EPS);
                double r = 1.0 / d;
                double v = r * w;
                m[0] += v; m[1] = fma(v, ty, m[1]); m[2] = fma(v, tx, m[2]); m[3] = fma(v, w, m[3]);
                double v2 = v * v;
                m[4] += v2; m[5] = fma(v2, ty, m[5]); m[6] = fma(v2, tx, m[6]); m[7] = fma(v2, w, m[7]);
                m[8] = fma(v2, ty * ty, m[8]); m[9] = fma(v2, tx * tx, m[9]);
                m[10] = fma(v2, w * ty, m[10]); m[11] = fma(v2, w * tx, m[11]); m[12] = fma(v2, w * w, m[12]);
                ob += log(d);
            }
#pragma unroll
            for (int i = 0; i < 13; i++) acc_add(acc, 27 + i, m[i]);
            acc_add(acc, NMOM, ob);
        }
        {
            const double d0 = ld_volatile(&Kp->d[0]), d1 = ld_volatile(&Kp->d[1]);
            double m[5] = {0, 0, 0, 0, 0};
            double ob = 0.0;
            for (int j = sD + lane; j < tot; j += 32) {
                unsigned e = E[j];
                double p = P[e & 0x7FF], q = Q[e & 0x7FF];
                double w = p * q;
                double d = fma(w, fma(w, d1, d0), EPS);
                double r = 1.0 / d;
                double v = r * w;
                m[0] += v; m[1] = fma(v, w, m[1]);
                double v2 = v * v;
                m[2] += v2; m[3] = fma(v2, w, m[3]); m[4] = fma(v2, w * w, m[4]);
                ob += log(d);
            }
#pragma unroll
            for (int i = 0; i < 5; i++) acc_add(acc, 40 + i, m[i]);
            acc_add(acc, NMOM, ob);
        }
    }
}

// ----------------------------------------------------------- reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sums the lane accumulators across the warp into o (all lanes get the totals).
__device__ inline void reduce_pass(const double* acc, PassOut& o) {
    for (int i = 0; i < NMOM; i++) o.mom[i] = warp_sum(acc[i * 32]);
    o.obj = warp_sum(acc[NMOM * 32]);
}

__device__ inline void zero_acc(double* acc) {
    for (int i = 0; i < NACC; i++) acc[i * 32] = 0.0;
}

// ------------------------------------------------------------- pair SQP

enum : int { PASS_FP32_DIRECT = 0, PASS_FP32_DIFF = 1, PASS_FP64 = 2 };

struct PairEval {
    double f;       // objective at the evaluated point
    double g[9];
    double H[81];
};

// Evaluates f, g, H at x.  For PASS_FP32_DIFF, f = f_base - (sum log(d/d_base))/n
// with x_base the accepted point.  wsm is the warp's shared-memory block.
__device__ inline void evaluate(const CohortDev& co, const uint16_t* ent, const uint16_t* hdr,
                                int64_t n, int kind, const double* x, const double* x_base,
                                double f_base, int lane, char* wsm, PairEval& ev, PassOut& po) {
    double* acc = reinterpret_cast<double*>(wsm) + lane;
    void* kbuf = wsm + WARP_SMEM_ACC;
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
    zero_acc(acc);
    __syncwarp();
    if (kind == PASS_FP64) {
        pass_fp64(co, ent, hdr, reinterpret_cast<const PassCoef*>(kbuf), acc, lane);
    } else if (kind == PASS_FP32_DIFF) {
        pass_fp32<OBJ_DIFF>(co, ent, hdr, reinterpret_cast<const Coef32*>(kbuf), acc, lane);
    } else {
        pass_fp32<OBJ_DIRECT>(co, ent, hdr, reinterpret_cast<const Coef32*>(kbuf), acc, lane);
    }
    __syncwarp();
    reduce_pass(acc, po);
    const double inv_n = 1.0 / (double)n;
    double S[9];
    rebuild(po.mom, S, ev.H);
    for (int i = 0; i < 9; i++) ev.g[i] = -S[i] / (double)n;
    for (int i = 0; i < 81; i++) ev.H[i] = ev.H[i] / (double)n;
    if (kind == PASS_FP64) {
        ev.f = -po.obj / (double)n;
    } else if (kind == PASS_FP32_DIRECT) {
        ev.f = -(po.obj * 0.69314718055994530942) * inv_n;
    } else {
        ev.f = f_base - po.obj * inv_n;
    }
}

constexpr double COND_RECHECK = 1e4;   // FP32 condition estimates above this are redone in FP64
constexpr double DIFF_BELOW = 1e-4;    // |alpha g.p| under which the objective change is summed directly

struct PairResult {
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
// FMA as 2 and a MUFU op as 1: the direct pass, and the extra of the
// log(d_new/d_old) objective.  Read off the loops of pass_fp32.
__host__ __device__ constexpr int flops_direct(int s) {
    return s == 0 ? 50 : s == 1 ? 39 : s == 2 ? 39 : s == 3 ? 55 : 27;
}
__host__ __device__ constexpr int flops_diff_extra(int s) {
    return s == 0 ? 18 : s == 1 ? 16 : s == 2 ? 16 : s == 3 ? 18 : 14;
}

__device__ inline void solve_pair(const CohortDev& co, const uint16_t* ent, const uint16_t* hdr,
                                  int64_t n, bool self_pair, int precision, const Tune& tu, int lane,
                                  char* wsm, PairResult& res) {
    double x[9];
    for (int i = 0; i < 9; i++) x[i] = self_pair ? 0.0 : 1.0 / 9.0;
    if (self_pair) { x[0] = 0.5; x[6] = 0.5; }
    normalise9(x);
    bool fp64 = (precision == 1);
    res.fp64_passes = 0;
    res.gh_passes = 0;
    res.obj_passes = 0;
    res.diff_passes = 0;
    res.escalated = false;
    PairEval ev;
    PassOut po;
    evaluate(co, ent, hdr, n, fp64 ? PASS_FP64 : PASS_FP32_DIRECT, x, x, 0.0, lane, wsm, ev, po);
    res.obj_passes++;
    res.gh_passes++;
    if (fp64) res.fp64_passes++;
    double f = ev.f;
    double g[9], H[81];
    for (int i = 0; i < 9; i++) g[i] = ev.g[i];
    for (int i = 0; i < 81; i++) H[i] = ev.H[i];
    int near_count = 0;
    for (uint64_t it = 0; it < tu.sqp_max_iter; it++) {
        double resid;
        bool conv = kkt_ok(x, g, tu.sqp_conv_tol, &resid);
        if (!fp64 && (conv || resid < 1e-6)) {
            if (!conv) near_count++;
            double cond = conv ? condition_estimate(x, g, H, tu.sqp_conv_tol) : 0.0;
            bool recheck = conv ? !(cond <= COND_RECHECK) : (near_count >= 3);
            if (recheck) {
                // FP64 re-evaluation at the same point; the pair stays FP64 from here.
                evaluate(co, ent, hdr, n, PASS_FP64, x, x, f, lane, wsm, ev, po);
                res.fp64_passes++;
                res.gh_passes++;
                res.obj_passes++;
                fp64 = true;
                res.escalated = true;
                f = ev.f;
                for (int i = 0; i < 9; i++) g[i] = ev.g[i];
                for (int i = 0; i < 81; i++) H[i] = ev.H[i];
                conv = kkt_ok(x, g, tu.sqp_conv_tol, &resid);
            } else if (conv) {
                for (int i = 0; i < 9; i++) res.x[i] = x[i];
                res.f = f;
                res.iters = it;
                res.cond = cond;
                return;
            }
        }
        if (conv) {
            for (int i = 0; i < 9; i++) res.x[i] = x[i];
            res.f = f;
            res.iters = it;
            res.cond = condition_estimate(x, g, H, tu.sqp_conv_tol);
            return;
        }
        // QP step: c = g - H x
        double c[9], y[9], p[9];
        for (int i = 0; i < 9; i++) c[i] = g[i] - dot_fma(9, H + i * 9, x);
        qp_simplex(H, c, x, tu, y);
        for (int i = 0; i < 9; i++) p[i] = y[i] - x[i];
        double gp = dot_fma(9, g, p);
        double tt = tu.bls_sufficient_decrease * gp;
        double alpha = 1.0;
        double xn[9];
        for (int bls = 0;;) {
            for (int i = 0; i < 9; i++) xn[i] = x[i] + alpha * p[i];
            normalise9(xn);
            int kind = fp64 ? PASS_FP64
                            : (fabs(alpha * gp) < DIFF_BELOW ? PASS_FP32_DIFF : PASS_FP32_DIRECT);
            evaluate(co, ent, hdr, n, kind, xn, x, f, lane, wsm, ev, po);
            res.obj_passes++;
            res.gh_passes++;
            if (kind == PASS_FP64) res.fp64_passes++;
            if (kind == PASS_FP32_DIFF) res.diff_passes++;
            bool accept = ev.f <= f + alpha * tt;
            bls++;
            if (accept || bls == tu.bls_max_iter) break;
            alpha *= tu.bls_step_size_reduce;
        }
        for (int i = 0; i < 9; i++) x[i] = xn[i];
        f = ev.f;
        for (int i = 0; i < 9; i++) g[i] = ev.g[i];
        for (int i = 0; i < 81; i++) H[i] = ev.H[i];
    }
    for (int i = 0; i < 9; i++) res.x[i] = x[i];
    res.f = f;
    res.iters = tu.sqp_max_iter;
    res.cond = CUDART_NAN;
}

}  // namespace kg
