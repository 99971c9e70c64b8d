// kg_wave.cu — wave kernels (admit / pass / solve) and their host loop.
// See kg_wave.cuh for the scheme; the SQP logic restates src/sqp.rs:49-310.
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>

#include "kg_engine.h"
#include "kg_bulk.cuh"
#include "kg_qp1.cuh"
#include "kg_wave.cuh"

namespace kg {

#define KG_WAVE_TRY(expr)                                                       \
    do {                                                                        \
        cudaError_t e_ = (expr);                                                \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);           \
            return e_ == cudaErrorMemoryAllocation ? KG_ENOMEM : KG_ECUDA;      \
        }                                                                       \
    } while (0)

constexpr int WAVE_WPB = 4;   // warps per block of the three wave kernels

// ------------------------------------------------------------------ admit

constexpr int ADMIT_WARPS = 8;   // warps that build one pair's lists together
constexpr int ADMIT_WARP_SMEM = UNIT_SITES * 4 + 6 * 32 * 4;   // FP32 output buffer, lane write positions


// Writes the frequency value t (p or 1 - p by the site's sel bit) of every
// jointly observed site of units [u0, u1) into its shape list, in site order,
// starting at off[] in each list.  Lane l owns word l of a unit (sites 32 l ..
// 32 l + 31): it forms the exclusive prefix of the shape counts over the lanes,
// then steps through its 32 bits in lockstep with the other lanes (no
// divergence).  The frequencies are read from the unit-transposed arrays, so
// each step's 32 lanes read 32 consecutive values (L1/L2 hits: every pair
// reads the same ones); FP32 values go through a shared output buffer so the
// global stores are coalesced, FP64 values are stored directly.
template <class T>
__device__ inline void scatter_lockstep(const CohortDev& co, int64_t x, int64_t y, int lane, int u0, int u1,
                                        const int64_t* off0, T* lists, char* wsm) {
    const uint2* px = co.planes_x + x * co.plane_stride;
    const uint2* py = co.planes_y + y * co.plane_stride;
    float* obuf = reinterpret_cast<float*>(wsm);   // FP32 only
    int off[5];
#pragma unroll
    for (int k = 0; k < 5; k++) off[k] = (int)off0[k];
    for (int u = u0; u < u1; u++) {
        const uint2 X = px[u * UNIT_WORDS + lane], Y = py[u * UNIT_WORDS + lane];
        // the unit's REF frequencies, unit-transposed: site 32 lane + i at
        // [32 i + lane], so step i of the lanes reads 32 consecutive values
        const T* freq = (sizeof(T) == 4 ? reinterpret_cast<const T*>(co.p32) : reinterpret_cast<const T*>(co.p64)) +
                        (int64_t)u * UNIT_SITES;
        const ShapeMasks sm = shape_masks(X, Y);
        unsigned c0 = sm.m[0] | sm.m[2] | sm.m[4];   // A 1, B1 2, B2 3, C 4, D 5
        unsigned c1 = sm.m[1] | sm.m[2];
        unsigned c2 = sm.m[3] | sm.m[4];
        unsigned sl = sm.sel;
        unsigned long long v = 0;
#pragma unroll
        for (int k = 0; k < 5; k++) v |= (unsigned long long)__popc(sm.m[k]) << (11 * k);
        unsigned long long inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        const unsigned long long tot = __shfl_sync(0xffffffffu, inc, 31);
        // unit-local write positions: shape starts in the unit plus this lane's prefix
        unsigned long long ust = 0;
        {
            unsigned acc = 0;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                ust |= (unsigned long long)acc << (11 * k);
                acc += (unsigned)((tot >> (11 * k)) & 0x7FFull);
            }
        }
        __syncwarp();
        if (sizeof(T) == 4) {
            // Branch-free: each site has a field index f (A 0, B1 1, B2 2, C 3,
            // D 4, not jointly observed 5) and the lane's write position for
            // each field sits in shared memory (counters[f][lane]): a site
            // writes at its field's position and advances it by its observed
            // bit.  Field 5 stays at 1023, which no list value of the unit
            // uses unless all 1,024 sites are observed, when field 5 is never
            // taken.  (Positions kept as 13-bit fields of one 64-bit register
            // cost 2% more admit time in 64-bit shifts.)  The 32 steps are
            // unrolled, so every shift count is a constant, and the list
            // offsets are 32-bit (a slot's lists hold far fewer than 2^31
            // entries), which keeps the loop's registers within the four
            // blocks per SM that the kernel needs (three ran 25% slower).
            const unsigned obs = sm.m[0] | sm.m[1] | sm.m[2] | sm.m[3] | sm.m[4];
            const unsigned f0 = sm.m[1] | sm.m[3] | ~obs, f1 = sm.m[2] | sm.m[3], f2 = sm.m[4] | ~obs;
            const unsigned long long pre = ust + (inc - v);
            int* cnt = reinterpret_cast<int*>(wsm + UNIT_SITES * 4) + lane;
#pragma unroll
            for (int k = 0; k < 5; k++) cnt[32 * k] = (int)((pre >> (11 * k)) & 0x7FFull);
            cnt[32 * 5] = 1023;
            const float* st = reinterpret_cast<const float*>(freq);
#pragma unroll
            for (int i = 0; i < 32; i++) {
                const unsigned f = ((f0 >> i) & 1u) | (((f1 >> i) & 1u) << 1) | (((f2 >> i) & 1u) << 2);
                int* c = cnt + 32 * f;
                const int pos = *c;
                *c = pos + (int)((obs >> i) & 1u);
                const float p = __ldg(st + i * 32 + lane);
                obuf[pos] = ((sl >> i) & 1u) ? 1.0f - p : p;
            }
        }
        unsigned long long Q = inc - v;
#pragma unroll
        for (int i = 0; i < (sizeof(T) == 4 ? 0 : 32); i++) {
            const int code = (int)((c0 & 1u) | ((c1 & 1u) << 1) | ((c2 & 1u) << 2));
            const bool flip = (sl & 1u) != 0;
            c0 >>= 1; c1 >>= 1; c2 >>= 1; sl >>= 1;
            if (code) {
                const int sh = 11 * (code - 1);
                const int pos = (int)((Q >> sh) & 0x7FFull);
                Q += 1ull << sh;
                const T p = __ldg(freq + i * 32 + lane);
                const T t = flip ? (T)1 - p : p;
                if (sizeof(T) == 4) {
                    obuf[pos] = (float)t;
                } else {
                    const int k = code - 1;
                    const int o = k == 0 ? off[0] : k == 1 ? off[1] : k == 2 ? off[2] : k == 3 ? off[3] : off[4];
                    lists[o + pos] = t;
                }
            }
        }
        __syncwarp();
        if (sizeof(T) == 4) {
            unsigned a = 0;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                const unsigned nk = (unsigned)((tot >> (11 * k)) & 0x7FFull);
                float* dst = reinterpret_cast<float*>(lists) + off[k];
                const float* srcb = obuf + a;
                for (unsigned j = lane; j < nk; j += 32) dst[j] = srcb[j];
                a += nk;
            }
            __syncwarp();
        }
#pragma unroll
        for (int k = 0; k < 5; k++) off[k] += (int)((tot >> (11 * k)) & 0x7FFull);
    }
}

// Each warp of the block takes a contiguous eighth of the pair's 1024-site
// units: it counts its sites per shape, the block turns the counts into write
// offsets (so the lists stay in site order), and each warp scatters its units.
// The returned count n also takes the pair's jointly called tri- and
// tetra-allelic sites (ML path), whose sums the multi-allelic kernel forms
// from the samples' reduced genotypes without a list.
template <class T>
__device__ inline int64_t build_lists(const CohortDev& co, int64_t x, int64_t y, T* lists, char* wsm,
                                      unsigned (*cnt)[6], int64_t* start, int64_t* count) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int u0 = (int)((int64_t)co.n_units * w / ADMIT_WARPS);
    const int u1 = (int)((int64_t)co.n_units * (w + 1) / ADMIT_WARPS);
    {
        const uint2* px = co.planes_x + x * co.plane_stride;
        const uint2* py = co.planes_y + y * co.plane_stride;
        unsigned c[5] = {0, 0, 0, 0, 0};
        for (int wd = u0 * UNIT_WORDS + lane; wd < u1 * UNIT_WORDS; wd += 32) {
            ShapeMasks sm = shape_masks(px[wd], py[wd]);
#pragma unroll
            for (int k = 0; k < 5; k++) c[k] += __popc(sm.m[k]);
        }
#pragma unroll
        for (int k = 0; k < 5; k++) {
            unsigned v = c[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) cnt[w][k] = v;
        }
        unsigned cm = 0;
        if (co.ml_nk > 0) {
            const int nw = co.ml_stride >> 5;
            const uint32_t* ox = co.ml_obs + x * nw;
            const uint32_t* oy = co.ml_obs + y * nw;
            for (int wd = w * 32 + lane; wd < nw; wd += ADMIT_WARPS * 32) cm += __popc(ox[wd] & oy[wd]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cm += __shfl_xor_sync(0xffffffffu, cm, o);
        }
        if (lane == 0) cnt[w][5] = cm;
    }
    __syncthreads();
    int64_t off[5], st = 0, n = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        int64_t tot = 0, before = 0;
        for (int v = 0; v < ADMIT_WARPS; v++) {
            if (v < w) before += cnt[v][k];
            tot += cnt[v][k];
        }
        start[k] = st;
        count[k] = tot;
        off[k] = st + before;
        st = align4(st + tot);
        n += tot;
    }
    if (n > 0) scatter_lockstep<T>(co, x, y, lane, u0, u1, off, lists, wsm);
    for (int v = 0; v < ADMIT_WARPS; v++) n += cnt[v][5];
    __syncthreads();   // cnt is reused by the block's next pair
    return n;
}

extern "C" __global__ void __launch_bounds__(ADMIT_WARPS * 32, 4) wave_admit_kernel(WaveArgs A) {
    __shared__ int sh_e;
    __shared__ unsigned long long sh_k;
    __shared__ unsigned cnt[ADMIT_WARPS][6];
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    char* wsm = smem + w * ADMIT_WARP_SMEM;
    if (A.clk->stop) return;   // a device loop past its last wave
    if (threadIdx.x == 0) atomicMin(&A.clk->start[0], global_ns());
    const PhaseEnd pe{&A.clk->end[0], threadIdx.x == 0};
    const int nfree = A.wc_cur->n_free;
    for (;;) {
        if (threadIdx.x == 0) sh_e = atomicAdd(A.admit_task, 1);
        __syncthreads();
        const int e = sh_e;
        __syncthreads();
        if (e >= nfree) return;
        const int s = A.free_cur[e];
        SlotState& S = A.slots[s];
        void* lists = A.lists + (int64_t)s * A.list_stride;
        int64_t start[5], count[5];
        if (S.status == SLOT_RESORT) {
            // an escalated pair: the same lists again, in FP64
            build_lists<double>(A.cohorts[S.cohort], S.x, S.y, static_cast<double*>(lists), wsm, cnt, start,
                                count);
            if (threadIdx.x == 0) {
                S.lists64 = 1;
                S.status = SLOT_PASS;
            }
            __syncthreads();
            if (w == 0) enqueue_pass<32>(A.pass_cur, A.tasks_cur, A.task_cap, A.wc_cur, s, S, lane, 0xffffffffu, A.unit_elems);
            continue;
        }
        // a free slot takes pairs until one has jointly observed sites
        for (;;) {
            if (threadIdx.x == 0) sh_k = atomicAdd(A.queue, 1ull);
            __syncthreads();
            const unsigned long long k = sh_k;
            __syncthreads();
            if (k >= (unsigned long long)A.live->total_pairs) {
                // no pair left for now: the slot waits in the next free list
                if (threadIdx.x == 0) A.free_next[atomicAdd(&A.wc_next->n_free, 1)] = s;
                break;
            }
            int c;
            int64_t j, x, y;
            decode_pair(A, (int64_t)k, c, j, x, y);
            const CohortDev& co = A.cohorts[c];
            const bool f64 = (A.precision == 1);
            const int64_t n = f64 ? build_lists<double>(co, x, y, static_cast<double*>(lists), wsm, cnt, start, count)
                                  : build_lists<float>(co, x, y, static_cast<float*>(lists), wsm, cnt, start, count);
            if (n == 0) {
                if (w == 0) {
                    double nan9[9];
                    for (int i = 0; i < 9; i++) nan9[i] = CUDART_NAN;
                    write_row(co.out + j, x, y, nan9, CUDART_NAN, 0, CUDART_NAN, lane);
                    if (lane == 0) {
                        atomicAdd(&A.counters->nosite_pairs, 1ull);
                        atomicAdd(&A.cohort_done[c], 1ull);
                    }
                }
                continue;
            }
            if (threadIdx.x == 0) {
                S.k = (int64_t)k;
                S.x = x;
                S.y = y;
                S.cohort = c;
                for (int i = 0; i < 5; i++) { S.start[i] = start[i]; S.cnt[i] = count[i]; }
                S.n = n;
                units_from_counts(S, A.unit_elems);
                S.lists64 = f64 ? 1 : 0;
                S.fp64 = f64 ? 1 : 0;
                S.near_count = 0;
                S.bls = 0;
                S.escalated = 0;
                S.gh = 0;
                S.f64p = 0;
                S.diffp = 0;
                S.it = 0;
                const bool self_pair = (co.kind == COHORT_TRIANGLE) && (x == y);
                double x0[9];
                for (int i = 0; i < 9; i++) x0[i] = self_pair ? 0.0 : 1.0 / 9.0;
                if (self_pair) { x0[0] = 0.5; x0[6] = 0.5; }
                normalise9(x0);
                for (int i = 0; i < 9; i++) { S.xc[i] = x0[i]; S.xt[i] = x0[i]; }
                S.f = 0.0;
                S.ev = EV_INIT;
                if (co.method == ESTIMATOR_CLS) set_coefficients(S, f64 ? PASS_CLS64 : PASS_CLS);
                else set_coefficients(S, f64 ? PASS_FP64 : PASS_FP32_DIRECT);
                S.status = SLOT_PASS;
            }
            __syncthreads();
            if (w == 0) enqueue_pass<32>(A.pass_cur, A.tasks_cur, A.task_cap, A.wc_cur, s, S, lane, 0xffffffffu, A.unit_elems);
            break;
        }
    }
}

// ------------------------------------------------------------------- pass

// Each pass warp streams its FP32 lists through a ring of RING_STAGES stages
// in its shared memory: lane 0 keeps up to RING_STAGES bulk copies in flight,
// so the site arithmetic reads shared memory while HBM fills the stages ahead.
constexpr int RING_STAGES = 4;
constexpr int STAGE_F4 = 128;                 // float4 per stage: four per lane
constexpr int STAGE_ELEMS = STAGE_F4 * 4;     // list entries per stage
static_assert(RING_STAGES * STAGE_F4 * 16 <= WARP_SMEM_BUF, "ring must fit the warp's buffer");
static_assert(sizeof(Coef32) + RING_STAGES * 8 <= WARP_SMEM_COEF, "coefficients and barriers must fit");

struct Ring {
    float4* buf;      // RING_STAGES * STAGE_F4
    uint64_t* bar;    // RING_STAGES barriers
    uint32_t seq;     // stages this warp has consumed so far
};

__device__ __forceinline__ void ring_issue(const Ring& R, const float* L, int64_t len, int i, uint32_t slot) {
    const int64_t e0 = (int64_t)i * STAGE_ELEMS;
    const int64_t ne = min((int64_t)STAGE_ELEMS, len - e0);
    const uint32_t bytes = (uint32_t)((ne * 4 + 15) & ~int64_t(15));
    bulk_load(R.buf + slot * STAGE_F4, L + e0, bytes, &R.bar[slot]);
}

// Lane 0 starts the first RING_STAGES stage copies of a list of len entries.
__device__ __forceinline__ void ring_prologue(const Ring& R, const float* L, int64_t len, int lane) {
    if (lane == 0) {
        const int nst = (int)((len + STAGE_ELEMS - 1) / STAGE_ELEMS);
        const int pro = min(nst, RING_STAGES);
        fence_proxy_async_smem();
        for (int i = 0; i < pro; i++) ring_issue(R, L, len, i, (R.seq + i) % RING_STAGES);
    }
}


// One shape's FP32 list from the ring.  Stage i holds float4 128 i .. 128 i +
// 127; lane l takes 128 i + 32 j + l (j = 0..3): 16 sites, in packed pairs
// (Shape32x2), whose FP32 gradient and objective partials go to FP64 after
// every stage (8 sites per partial) and whose Hessian partials go every
// HESS_STAGES stages (128 sites per partial).  Only the list's last stage can
// be partly filled; the others run without bounds tests.  L and every stage
// start are 16-byte aligned (list starts are multiples of four entries); a
// stage's copy rounds its size up to 16 bytes, which stays inside the slot's
// list buffer.  The FP64 Hessian sums live in the warp's shared memory (Hs,
// moment j of lane l at Hs[32 j + l]), which leaves registers for a fifth
// block per SM.  The sums use the hi coefficients only (lo_correction
// restores the rest).  A stage is read with plain shared-memory loads: the
// barrier wait (a memory clobber) keeps them after the copy has landed and
// the warp sync keeps them before the stage's next copy, and between the two
// the compiler schedules them among the site arithmetic.  Returns false if a
// wait ran out.
constexpr int HESS_STAGES = 16;
template <int S, bool DIFF>
__device__ __forceinline__ bool stream32_ring(const float* __restrict__ L, int64_t len, const Coef32* K, int lane,
                                              const Ring R, double* Hs, LaneSums& out) {
    using E = Shape32x2<S>;
    constexpr int NG = E::NG, NH = E::NH, GOFF = E::GOFF, HOFF = E::HOFF;
    E ev;
    ev.load(K, DIFF);
    double G[NG], F = 0.0;
    double* H = Hs + lane;
    float2 h[NH];
#pragma unroll
    for (int i = 0; i < NG; i++) G[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NH; i++) { H[32 * i] = 0.0; h[i] = dup2(0.f); }
    const int64_t n4 = len >> 2;
    const int nst = (int)((len + STAGE_ELEMS - 1) / STAGE_ELEMS);
    const int nfull = (int)(n4 / STAGE_F4);   // stages with all 128 float4 inside the list
    const uint32_t seq0 = R.seq;   // ring_prologue has issued the first stages
    bool ok = true;
    int done = 0;
    for (int i = 0; i < nst; i++) {
        const uint32_t q = seq0 + i;
        const uint32_t slot = q % RING_STAGES;
        if (!mbar_wait(&R.bar[slot], (q / RING_STAGES) & 1u)) { ok = false; break; }
        done = i + 1;
        const float4* B4 = R.buf + slot * STAGE_F4 + lane;
        float2 g[NG], o = dup2(0.f);
#pragma unroll
        for (int j = 0; j < NG; j++) g[j] = dup2(0.f);
        if (i < nfull) {
#pragma unroll
            for (int j = 0; j < 4; j++) ev.template site4<DIFF>(B4[32 * j], g, o, h, j & 1);
        } else {
            const int rem = (int)(n4 - (int64_t)i * STAGE_F4);   // float4 in this stage, 0..127
#pragma unroll
            for (int j = 0; j < 4; j++)
                if (lane + 32 * j < rem) ev.template site4<DIFF>(B4[32 * j], g, o, h, j & 1);
        }
#pragma unroll
        for (int j = 0; j < NG; j++) { G[j] += (double)g[j].x; G[j] += (double)g[j].y; }
        F += (double)o.x;
        F += (double)o.y;
        if (i % HESS_STAGES == HESS_STAGES - 1) {
#pragma unroll
            for (int j = 0; j < NH; j++) { H[32 * j] += (double)(h[j].x + h[j].y); h[j] = dup2(0.f); }
        }
        if (i + RING_STAGES < nst) {
            __syncwarp();
            if (lane == 0) {
                fence_proxy_async_smem();
                ring_issue(R, L, len, i + RING_STAGES, slot);
            }
        }
    }
    if (!ok) {
        // let this warp's copies in flight land before it leaves
        const int issued = min(nst, done + RING_STAGES);
        for (int i = done; i < issued; i++) {
            const uint32_t q = seq0 + i;
            if (!mbar_wait(&R.bar[q % RING_STAGES], (q / RING_STAGES) & 1u)) break;
        }
        return false;
    }
    double Hf[NH];
#pragma unroll
    for (int j = 0; j < NH; j++) Hf[j] = H[32 * j] + (double)(h[j].x + h[j].y);
    if (lane < (int)(len & 3)) {
        // the last len % 4 entries, one site per lane
        Shape32<S, false> es;
        es.load(K, DIFF);
        const float* B = reinterpret_cast<const float*>(R.buf + ((seq0 + nst - 1) % RING_STAGES) * STAGE_F4);
        float g[NG], hs[NH], ob = 0.f;
#pragma unroll
        for (int j = 0; j < NG; j++) g[j] = 0.f;
#pragma unroll
        for (int j = 0; j < NH; j++) hs[j] = 0.f;
        es.site(B[4 * n4 - (int64_t)(nst - 1) * STAGE_ELEMS + lane], g, ob, hs);
#pragma unroll
        for (int j = 0; j < NG; j++) G[j] += (double)g[j];
#pragma unroll
        for (int j = 0; j < NH; j++) Hf[j] += (double)hs[j];
        F += (double)ob;
    }
    __syncwarp();   // every lane has read the ring before the next copies
#pragma unroll
    for (int j = 0; j < NG; j++) out.m[GOFF + j] = G[j];
#pragma unroll
    for (int j = 0; j < NH; j++) out.m[HOFF + j] = Hf[j];
    out.obj += F;
    return true;
}

// ------------------------------------------------------------- CLS moments
// The CLS estimator's c needs the sums over a pair's sites of its likelihood
// rows, which are the ML gradient moments with r = 1: per shape sum t^k (A),
// sum w t^k (B1, B2), sum w {1, ty, t, w} (C) and sum w {1, w} (D).  One pass,
// no reciprocal and no logarithm; the same FP32 partials of 8 sites per half,
// promoted to FP64 (the Hessian and objective slots of the partials stay 0).
template <int S>
__device__ __forceinline__ void cls_pair(float2 t, float2* g) {
    if (S == 0) {
        const float2 t2 = mul2(t, t), t3 = mul2(t2, t);
        g[0] = add2(g[0], t); g[1] = fma2(t, t, g[1]); g[2] = fma2(t2, t, g[2]); g[3] = fma2(t3, t, g[3]);
    } else if (S == 1 || S == 2) {
        const float2 w = fma2(neg2(t), t, t), w1 = mul2(w, t);
        g[0] = add2(g[0], w); g[1] = fma2(w, t, g[1]); g[2] = fma2(w1, t, g[2]);
    } else if (S == 3) {
        const float2 ty = add2(dup2(1.0f), neg2(t)), w = mul2(t, ty);
        g[0] = add2(g[0], w); g[1] = fma2(w, ty, g[1]); g[2] = fma2(w, t, g[2]); g[3] = fma2(w, w, g[3]);
    } else {
        const float2 w = fma2(neg2(t), t, t);
        g[0] = add2(g[0], w); g[1] = fma2(w, w, g[1]);
    }
}

template <int S>
__device__ __forceinline__ void cls_site(float t, float* g) {
    if (S == 0) {
        const float t2 = t * t, t3 = t2 * t;
        g[0] += t; g[1] = fmaf(t, t, g[1]); g[2] = fmaf(t2, t, g[2]); g[3] = fmaf(t3, t, g[3]);
    } else if (S == 1 || S == 2) {
        const float w = fmaf(-t, t, t), w1 = w * t;
        g[0] += w; g[1] = fmaf(w, t, g[1]); g[2] = fmaf(w1, t, g[2]);
    } else if (S == 3) {
        const float ty = 1.0f - t, w = t * ty;
        g[0] += w; g[1] = fmaf(w, ty, g[1]); g[2] = fmaf(w, t, g[2]); g[3] = fmaf(w, w, g[3]);
    } else {
        const float w = fmaf(-t, t, t);
        g[0] += w; g[1] = fmaf(w, w, g[1]);
    }
}

// FP32 lists through the ring (the protocol of stream32_ring).
template <int S>
__device__ __forceinline__ bool cls_stream32_ring(const float* __restrict__ L, int64_t len, int lane, const Ring R,
                                                  LaneSums& out) {
    constexpr int NG = Shape32x2<S>::NG, NH = Shape32x2<S>::NH, GOFF = Shape32x2<S>::GOFF,
                  HOFF = Shape32x2<S>::HOFF;
    double G[NG];
#pragma unroll
    for (int i = 0; i < NG; i++) G[i] = 0.0;
    const int64_t n4 = len >> 2;
    const int nst = (int)((len + STAGE_ELEMS - 1) / STAGE_ELEMS);
    const int nfull = (int)(n4 / STAGE_F4);
    const uint32_t seq0 = R.seq;
    bool ok = true;
    int done = 0;
    for (int i = 0; i < nst; i++) {
        const uint32_t q = seq0 + i;
        const uint32_t slot = q % RING_STAGES;
        if (!mbar_wait(&R.bar[slot], (q / RING_STAGES) & 1u)) { ok = false; break; }
        done = i + 1;
        const float4* B4 = R.buf + slot * STAGE_F4 + lane;
        float2 g[NG];
#pragma unroll
        for (int j = 0; j < NG; j++) g[j] = dup2(0.f);
        const int rem = i < nfull ? STAGE_F4 : (int)(n4 - (int64_t)i * STAGE_F4);
#pragma unroll
        for (int j = 0; j < 4; j++)
            if (lane + 32 * j < rem) {
                const float4 v = B4[32 * j];
                cls_pair<S>(make_float2(v.x, v.y), g);
                cls_pair<S>(make_float2(v.z, v.w), g);
            }
#pragma unroll
        for (int j = 0; j < NG; j++) { G[j] += (double)g[j].x; G[j] += (double)g[j].y; }
        if (i + RING_STAGES < nst) {
            __syncwarp();
            if (lane == 0) {
                fence_proxy_async_smem();
                ring_issue(R, L, len, i + RING_STAGES, slot);
            }
        }
    }
    if (!ok) {
        const int issued = min(nst, done + RING_STAGES);
        for (int i = done; i < issued; i++) {
            const uint32_t q = seq0 + i;
            if (!mbar_wait(&R.bar[q % RING_STAGES], (q / RING_STAGES) & 1u)) break;
        }
        return false;
    }
    if (lane < (int)(len & 3)) {
        const float* B = reinterpret_cast<const float*>(R.buf + ((seq0 + nst - 1) % RING_STAGES) * STAGE_F4);
        float g[NG];
#pragma unroll
        for (int j = 0; j < NG; j++) g[j] = 0.f;
        cls_site<S>(B[4 * n4 - (int64_t)(nst - 1) * STAGE_ELEMS + lane], g);
#pragma unroll
        for (int j = 0; j < NG; j++) G[j] += (double)g[j];
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < NG; j++) out.m[GOFF + j] = G[j];
#pragma unroll
    for (int j = 0; j < NH; j++) out.m[HOFF + j] = 0.0;
    return true;
}

// FP64 lists (the FP64 form): the same moments in FP64, read directly.
template <int S>
__device__ __noinline__ void cls_stream64(const double* __restrict__ L, int64_t len, int lane, LaneSums& out) {
    constexpr int NG = Shape32x2<S>::NG, NH = Shape32x2<S>::NH, GOFF = Shape32x2<S>::GOFF,
                  HOFF = Shape32x2<S>::HOFF;
    double g[NG];
#pragma unroll
    for (int i = 0; i < NG; i++) g[i] = 0.0;
    for (int64_t i = lane; i < len; i += 32) {
        const double t = L[i];
        if (S == 0) {
            const double t2 = t * t, t3 = t2 * t;
            g[0] += t; g[1] = fma(t, t, g[1]); g[2] = fma(t2, t, g[2]); g[3] = fma(t3, t, g[3]);
        } else if (S == 1 || S == 2) {
            const double w = t * (1.0 - t), w1 = w * t;
            g[0] += w; g[1] = fma(w, t, g[1]); g[2] = fma(w1, t, g[2]);
        } else if (S == 3) {
            const double ty = 1.0 - t, w = t * ty;
            g[0] += w; g[1] = fma(w, ty, g[1]); g[2] = fma(w, t, g[2]); g[3] = fma(w, w, g[3]);
        } else {
            const double w = t * (1.0 - t);
            g[0] += w; g[1] = fma(w, w, g[1]);
        }
    }
#pragma unroll
    for (int j = 0; j < NG; j++) out.m[GOFF + j] = g[j];
#pragma unroll
    for (int j = 0; j < NH; j++) out.m[HOFF + j] = 0.0;
}

template <int SH>
__device__ __forceinline__ bool run_unit(const void* lists, bool l64, int64_t off, int64_t len,
                                         const void* kbuf, bool diff, int lane, const Ring R, double* Hs,
                                         LaneSums& ls, bool cls) {
    if (cls) {
        if (l64) {
            cls_stream64<SH>(static_cast<const double*>(lists) + off, len, lane, ls);
            return true;
        }
        return cls_stream32_ring<SH>(static_cast<const float*>(lists) + off, len, lane, R, ls);
    }
    if (l64) {
        stream64<SH>(static_cast<const double*>(lists) + off, len, reinterpret_cast<const PassCoef*>(kbuf),
                     lane, ls);
        return true;
    }
    const float* L = static_cast<const float*>(lists) + off;
    const Coef32* K = reinterpret_cast<const Coef32*>(kbuf);
    return diff ? stream32_ring<SH, true>(L, len, K, lane, R, Hs, ls)
                : stream32_ring<SH, false>(L, len, K, lane, R, Hs, ls);
}

// Five blocks of four warps per SM (at most 102 registers a thread).  Each
// warp's shared memory: the list ring, the pass coefficients with the ring's
// barriers, and the FP64 Hessian sums of its lanes.
constexpr int PASS_MIN_BLOCKS = 5;
constexpr int PASS_HESS_BYTES = 9 * 32 * 8;
constexpr int PASS_WARP_SMEM = WARP_SMEM + PASS_HESS_BYTES;
extern "C" __global__ void __launch_bounds__(128, PASS_MIN_BLOCKS) wave_pass_kernel(WaveArgs A) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    char* wsm = smem + wib * PASS_WARP_SMEM;
    char* kbuf = wsm + WARP_SMEM_BUF;
    double* hsm = reinterpret_cast<double*>(wsm + WARP_SMEM);
    if (A.clk->stop) return;   // a device loop past its last wave
    if (threadIdx.x == 0) atomicMin(&A.clk->start[1], global_ns());
    const PhaseEnd pe{&A.clk->end[1], lane == 0};
    Ring R;
    R.buf = reinterpret_cast<float4*>(wsm);
    R.bar = reinterpret_cast<uint64_t*>(kbuf + sizeof(Coef32));
    R.seq = 0;
    if (lane == 0) {
        for (int i = 0; i < RING_STAGES; i++) mbar_init(&R.bar[i], 1);
        fence_mbar_init();
    }
    __syncwarp();
    int pre[6];
    pre[0] = 0;
#pragma unroll
    for (int k = 0; k < 5; k++) pre[k + 1] = pre[k] + A.wc_cur->units[k] + A.wc_cur->back[k];
    const int64_t ntask = pre[5];
    // the next task is claimed as the current one starts, so the claim's
    // latency hides behind the current task's sites
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(A.pass_task, 1ull);
    t = __shfl_sync(0xffffffffu, t, 0);
    for (;;) {
        if ((int64_t)t >= ntask) break;
        int sh = 0;
#pragma unroll
        for (int k = 1; k < 5; k++) sh += ((int)t >= pre[k]) ? 1 : 0;
        const int jt = (int)t - pre[sh], nfront = A.wc_cur->units[sh];
        const int4 tk = A.tasks_cur[sh * A.task_cap + (jt < nfront ? (int64_t)jt : A.task_cap - 1 - (jt - nfront))];
        unsigned long long t_next = 0;
        if (lane == 0) t_next = atomicAdd(A.pass_task, 1ull);
        const int s = tk.x;
        const int u = tk.y;
        const int64_t off = tk.z;
        const int64_t len = tk.w & 0xFFFFFF;
        const int kind = tk.w >> 24;
        const bool cls = (kind == PASS_CLS || kind == PASS_CLS64);
        const bool l64 = (kind == PASS_FP64 || kind == PASS_CLS64);
        const SlotState& S = A.slots[s];
        // first list stages in flight, then the pass's coefficients into shared memory
        if (!l64) ring_prologue(R, reinterpret_cast<const float*>(A.lists + (int64_t)s * A.list_stride) + off, len, lane);
        const int nwords = l64 ? (int)(sizeof(PassCoef) / 4) : (int)(sizeof(Coef32) / 4);
        const uint32_t* src = l64 ? reinterpret_cast<const uint32_t*>(&S.c64)
                                  : reinterpret_cast<const uint32_t*>(&S.c32);
        for (int w = lane; w < nwords; w += 32) reinterpret_cast<uint32_t*>(kbuf)[w] = src[w];
        __syncwarp();
        const void* lists = A.lists + (int64_t)s * A.list_stride;
        const bool diff = (kind == PASS_FP32_DIFF);
        LaneSums ls;
        ls.obj = 0.0;
        bool ok;
        switch (sh) {
        case 0: ok = run_unit<0>(lists, l64, off, len, kbuf, diff, lane, R, hsm, ls, cls); break;
        case 1: ok = run_unit<1>(lists, l64, off, len, kbuf, diff, lane, R, hsm, ls, cls); break;
        case 2: ok = run_unit<2>(lists, l64, off, len, kbuf, diff, lane, R, hsm, ls, cls); break;
        case 3: ok = run_unit<3>(lists, l64, off, len, kbuf, diff, lane, R, hsm, ls, cls); break;
        default: ok = run_unit<4>(lists, l64, off, len, kbuf, diff, lane, R, hsm, ls, cls); break;
        }
        if (!__all_sync(0xffffffffu, ok)) {
            if (lane == 0) atomicAdd(&A.counters->stalled_waits, 1ull);
            return;
        }
        if (!l64) R.seq += (uint32_t)((len + STAGE_ELEMS - 1) / STAGE_ELEMS);
        const int go = shape_goff(sh), nv = shape_ng(sh) + shape_nh(sh);
        double* P = A.partial + ((int64_t)s * A.max_units + u) * UNIT_VALS;
        for (int i = 0; i < nv; i++) {
            const double v = warp_sum(ls.m[go + i]);
            if (lane == 0) P[i] = v;
        }
        const double ob = warp_sum(ls.obj);
        if (lane == 0) P[UNIT_VALS - 1] = ob;
        __syncwarp();
        t = __shfl_sync(0xffffffffu, t_next, 0);
    }
}

// ------------------------------------------------- tri- and tetra-allelic

// The sums of the ML path's tri- and tetra-allelic sites for every slot with
// a pending ML pass: per kept site with both samples called, the row L =
// m[g'x][g'y] from the site's table, d = eps + L.xt, and the terms L/d
// (gradient), (L/d)(L/d)' (Hessian) and the objective term (log d, or for a
// difference pass log(d / d_old) with d_old at xc); a call that uses a
// dropped allele gives the site a row of zeros (objective term log eps, or 0
// in a difference pass).  Work units are (slot of the pass list, ml_chunk
// sites), strided over the grid's warps; lanes stride over the unit's sites,
// and the unit's sums go to ml_partial in a fixed order.
//
// FP32 passes evaluate as the biallelic passes do: the FP32 rows with the FP32
// hi parts of xt, FP32 partial sums added to the lane's FP64 sums in shared
// memory (gradient and objective every 8 sites, Hessian every 64), and the lo
// parts of xt restored to first order in FP64 from the unit's own sums (G_i
// loses sum_j H_ij lo_j, the objective gains sum_j lo_j G_j).  FP64 passes use
// the FP64 rows, their Hessian sums in the same shared memory.
constexpr int MULTI_WARPS = 4;
// shared-memory rows of a warp's sums (32 lane partials each): the 45 Hessian
// terms, the 9 gradient terms, the objective
constexpr int MULTI_HS_ROWS = 55;
// per lane MULTI_STAGES row slots of 48 bytes after the sums
constexpr int MULTI_STAGES = 3;
constexpr int MULTI_WARP_SMEM = MULTI_HS_ROWS * 32 * (int)sizeof(double) + 32 * MULTI_STAGES * 48;
constexpr int MULTI_SMEM = MULTI_WARPS * MULTI_WARP_SMEM;

// A lane's multi-allelic site as loaded: its two codes and table entry; then
// its row index (ML_ROW_NONE: a missing call, ML_ROW_ZERO: a call with a
// dropped allele, whose row is zero).
struct MultiCodes {
    int a, b;
    int2 si;
};
constexpr int ML_ROW_NONE = -1, ML_ROW_ZERO = -2;
__device__ __forceinline__ MultiCodes multi_codes(const CohortDev& co, const uint8_t* grx, const uint8_t* gry,
                                                  int64_t v, int64_t v1) {
    MultiCodes c{ML_MISSING, ML_MISSING, make_int2(0, 0)};
    if (v < v1) {
        c.a = grx[v];
        c.b = gry[v];
        c.si = co.ml_site[v];
    }
    return c;
}
__device__ __forceinline__ int multi_row_index(const MultiCodes& c) {
    if (c.a == ML_MISSING || c.b == ML_MISSING) return ML_ROW_NONE;
    if (c.a == ML_ZERO_ROW || c.b == ML_ZERO_ROW) return ML_ROW_ZERO;
    return c.si.x + c.a * c.si.y + c.b;
}

template <bool DIFF>
__device__ __forceinline__ void multi_unit32(const CohortDev& co, const SlotState& S, int64_t v0, int64_t v1,
                                             int lane, double eps, double* hs, double* P) {
    float xh[9], sd[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        xh[k] = (float)S.xt[k];
        sd[k] = DIFF ? (float)(S.xt[k] - S.xc[k]) : 0.f;
    }
    const uint8_t* grx = co.ml_gr + S.x * co.ml_stride;
    const uint8_t* gry = co.ml_gr + S.y * co.ml_stride;
    const float e32 = (float)eps;
    float g[9], h[45], o = 0.f;
#pragma unroll
    for (int k = 0; k < 9; k++) g[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 45; k++) h[k] = 0.f;
    int nzero = 0;
    for (int k = 0; k < MULTI_HS_ROWS; k++) hs[32 * k + lane] = 0.0;
    // Warp-uniform iterations, so that the FP64 flushes run once per warp.
    // Loads run ahead without holding registers: the codes three sites ahead
    // into registers, the row two sites ahead by cp.async into the lane's
    // MULTI_STAGES slots in shared memory (the row's address needs the codes).
    const int iters = (int)((v1 - v0 + 31) >> 5);
    float4* slots = reinterpret_cast<float4*>(hs + 32 * MULTI_HS_ROWS) + lane * (3 * MULTI_STAGES);
    const uint32_t slot0 = smem_u32(slots);
    auto issue_row = [&](int ri, int stage) {
        if (ri >= 0) {
            const float4* R = co.ml_rows32 + 3 * (int64_t)ri;
            const uint32_t d = slot0 + 48u * (uint32_t)stage;
            cp_async16(d, R);
            cp_async16(d + 16u, R + 1);
            cp_async16(d + 32u, R + 2);
        }
        cp_async_commit();
    };
    int ri0 = multi_row_index(multi_codes(co, grx, gry, v0 + lane, v1));
    int ri1 = multi_row_index(multi_codes(co, grx, gry, v0 + lane + 32, v1));
    issue_row(ri0, 0);
    issue_row(ri1, 1);
    MultiCodes c2 = multi_codes(co, grx, gry, v0 + lane + 64, v1);
    for (int it = 0; it < iters; it++) {
        const int ri2 = multi_row_index(c2);
        issue_row(ri2, (it + 2) % MULTI_STAGES);
        c2 = multi_codes(co, grx, gry, v0 + lane + 32 * (int64_t)(it + 3), v1);
        cp_async_wait<2>();   // this site's row has landed
        if (ri0 >= 0) {
            const float4* Rs = slots + 3 * (it % MULTI_STAGES);
            const float4 r0 = Rs[0], r1 = Rs[1], r2 = Rs[2];
            const float L[9] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w, r2.x};
            const float d = dot9_eps(L, xh, e32);
            const float r = rcp_approx(d);
            float q[9];
#pragma unroll
            for (int k = 0; k < 9; k++) {
                q[k] = L[k] * r;
                g[k] += q[k];
            }
            int hh = 0;
#pragma unroll
            for (int i = 0; i < 9; i++)
#pragma unroll
                for (int j = i; j < 9; j++, hh++) h[hh] = fmaf(q[i], q[j], h[hh]);
            if (!DIFF) {
                o += lg2_approx(d);
            } else {
                float dl = 0.f;
#pragma unroll
                for (int k = 0; k < 9; k++) dl = fmaf(L[k], sd[k], dl);
                o += neg_log1m(dl * r);
            }
        } else if (ri0 == ML_ROW_ZERO) {
            nzero++;
        }
        ri0 = ri1;
        ri1 = ri2;
        if ((it & 7) == 7) {
#pragma unroll
            for (int k = 0; k < 9; k++) {
                hs[32 * (45 + k) + lane] += (double)g[k];
                g[k] = 0.f;
            }
            hs[32 * 54 + lane] += (double)o;
            o = 0.f;
        }
        if ((it & 63) == 63) {
#pragma unroll
            for (int k = 0; k < 45; k++) {
                hs[32 * k + lane] += (double)h[k];
                h[k] = 0.f;
                asm volatile("" ::: "memory");   // one read-modify-write at a time: no register peak
            }
        }
    }
    cp_async_wait<0>();   // no copy outstanding into the slots (they are past the last site)
    // the partials leave the registers before the reductions
#pragma unroll
    for (int k = 0; k < 45; k++) hs[32 * k + lane] += (double)h[k];
#pragma unroll
    for (int k = 0; k < 9; k++) hs[32 * (45 + k) + lane] += (double)g[k];
    hs[32 * 54 + lane] += (double)o;
    double G[9], lo[9], corr[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        G[k] = warp_sum(hs[32 * (45 + k) + lane]);
        lo[k] = S.xt[k] - (double)xh[k];
        corr[k] = 0.0;
    }
    const double F = warp_sum(hs[32 * 54 + lane]);
    int hh = 0;
#pragma unroll
    for (int i = 0; i < 9; i++)
#pragma unroll
        for (int j = i; j < 9; j++, hh++) {
            const double t = warp_sum(hs[32 * hh + lane]);
            if (lane == 0) P[9 + hh] = t;
            corr[i] = fma(t, lo[j], corr[i]);
            if (j != i) corr[j] = fma(t, lo[i], corr[j]);
        }
    double ob;
    if (DIFF) {
        ob = F;
    } else {
        double c = 0.0;
#pragma unroll
        for (int k = 0; k < 9; k++) c = fma(lo[k], G[k], c);
        for (int off = 16; off > 0; off >>= 1) nzero += __shfl_xor_sync(0xffffffffu, nzero, off);
        ob = (F * 0.69314718055994530942 + c) + (double)nzero * log(eps);
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 9; k++) P[k] = G[k] - corr[k];
        P[54] = ob;
    }
    __syncwarp();
}

__device__ __forceinline__ void multi_unit64(const CohortDev& co, const SlotState& S, int64_t v0, int64_t v1,
                                             int lane, double eps, double* hs, double* P) {
    const bool diff = S.kind == PASS_FP32_DIFF;
    double xt[9], xc[9];
#pragma unroll
    for (int k = 0; k < 9; k++) { xt[k] = S.xt[k]; xc[k] = S.xc[k]; }
    const uint8_t* grx = co.ml_gr + S.x * co.ml_stride;
    const uint8_t* gry = co.ml_gr + S.y * co.ml_stride;
    double g[9], ob = 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) g[k] = 0.0;
    for (int k = 0; k < 45; k++) hs[32 * k + lane] = 0.0;
    for (int64_t v = v0 + lane; v < v1; v += 32) {
        const int a = grx[v], b = gry[v];
        if (a == ML_MISSING || b == ML_MISSING) continue;
        if (a == ML_ZERO_ROW || b == ML_ZERO_ROW) {
            if (!diff) ob += log(eps);
            continue;
        }
        const int2 si = co.ml_site[v];
        const double* R = co.ml_rows + 9 * ((int64_t)si.x + a * si.y + b);
        double L[9];
#pragma unroll
        for (int k = 0; k < 9; k++) L[k] = __ldg(R + k);
        double d = eps;
#pragma unroll
        for (int k = 0; k < 9; k++) d = fma(L[k], xt[k], d);
        const double r = 1.0 / d;
        double q[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            q[k] = L[k] * r;
            g[k] += q[k];
        }
        int h = 0;
#pragma unroll
        for (int i = 0; i < 9; i++)
#pragma unroll
            for (int j = i; j < 9; j++, h++) hs[32 * h + lane] = fma(q[i], q[j], hs[32 * h + lane]);
        if (!diff) {
            ob += log(d);
        } else {
            double dc = eps, dl = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++) {
                dc = fma(L[k], xc[k], dc);
                dl = fma(L[k], xt[k] - xc[k], dl);
            }
            ob += log1p(dl / dc);
        }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const double v = warp_sum(g[k]);
        if (lane == 0) P[k] = v;
    }
    for (int k = 0; k < 45; k++) {
        const double v = warp_sum(hs[32 * k + lane]);
        if (lane == 0) P[9 + k] = v;
    }
    const double vo = warp_sum(ob);
    if (lane == 0) P[54] = vo;
    __syncwarp();
}

extern "C" __global__ void __launch_bounds__(MULTI_WARPS * 32, 3) wave_multi_kernel(WaveArgs A) {
    extern __shared__ double multi_smem[];   // per warp MULTI_HS_ROWS x 32 lane sums
    if (A.clk->stop) return;   // a device loop past its last wave
    const int lane = threadIdx.x & 31;
    const PhaseEnd pe{&A.clk->end[1], lane == 0};   // timed as part of the pass phase
    const int64_t warp = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
    const int64_t ntask = (int64_t)A.wc_cur->n_pass * A.ml_units;
    const double eps = A.tune.epsilon;
    double* hs = multi_smem + (threadIdx.x >> 5) * (MULTI_WARP_SMEM / (int)sizeof(double));
    for (int64_t t = warp; t < ntask; t += nwarps) {
        const int s = A.pass_cur[t / A.ml_units];
        const int u = (int)(t % A.ml_units);
        const SlotState& S = A.slots[s];
        const int kind = S.kind;
        if (kind == PASS_CLS || kind == PASS_CLS64) continue;
        const CohortDev& co = A.cohorts[S.cohort];
        const int64_t v0 = (int64_t)u * A.ml_chunk;
        if (v0 >= co.ml_nk) continue;
        const int64_t v1 = min((int64_t)co.ml_nk, v0 + A.ml_chunk);
        double* P = A.ml_partial + ((int64_t)s * A.ml_units + u) * ML_VALS;
        if (kind == PASS_FP64) multi_unit64(co, S, v0, v1, lane, eps, hs, P);
        else if (kind == PASS_FP32_DIFF) multi_unit32<true>(co, S, v0, v1, lane, eps, hs, P);
        else multi_unit32<false>(co, S, v0, v1, lane, eps, hs, P);
    }
}

// Index of Hessian entry (i, j) in the upper triangle (row-major) of 9 x 9.
__device__ __forceinline__ int upper9(int i, int j) {
    const int a = i < j ? i : j, b = i < j ? j : i;
    return a * 9 - a * (a - 1) / 2 + (b - a);
}

// ------------------------------------------------------------------ solve

// (lane: the lane's index in its half-warp group)
__device__ inline void finish_slot(const WaveArgs& A, SlotState& S, int s, const double* x, double f,
                                   uint64_t iters, double cond, int lane) {
    const CohortDev& co = A.cohorts[S.cohort];
    const int64_t j = S.k - co.pair_begin;
    write_row(co.out + j, S.x, S.y, x, f, iters, cond, lane);
    if (lane == 0) {
        RunCounters* C = A.counters;
        atomicAdd(&C->gh_passes, (unsigned long long)S.gh);
        atomicAdd(&C->obj_passes, (unsigned long long)S.gh);
        atomicAdd(&C->fp64_passes, (unsigned long long)S.f64p);
        atomicAdd(&C->fp64_pairs, (unsigned long long)S.escalated);
        atomicAdd(&C->pair_sites, (unsigned long long)S.n);
        atomicAdd(&C->work_units, (unsigned long long)S.n * (unsigned long long)S.gh);
        if (iters >= co.max_iter) atomicAdd(&C->nonconverged, 1ull);
        const int p32 = co.method == ESTIMATOR_CLS ? 0 : S.gh - S.f64p;   // the ML site arithmetic only
        unsigned long long f32 = 0, f64 = 0;
        for (int sh = 0; sh < 5; sh++) {
            atomicAdd(&C->shape_sites[sh], (unsigned long long)S.cnt[sh]);
            f32 += (unsigned long long)S.cnt[sh] * (unsigned long long)(p32 * flops4_fp32_hi(sh) + S.diffp * flops4_diff_extra(sh));
            f64 += (unsigned long long)S.cnt[sh] * (unsigned long long)(S.f64p * flops_fp64(sh));
        }
        atomicAdd(&C->flops_fp32, f32 / 4);
        atomicAdd(&C->flops_fp64, f64);
        S.status = SLOT_FREE;
        A.free_next[atomicAdd(&A.wc_next->n_free, 1)] = s;
        atomicAdd(&A.cohort_done[S.cohort], 1ull);
    }
}

// A self pair's CLS problem: the two-variable QP on (Delta1, Delta7) from
// (1/2, 1/2) (src/coefficients.rs:231-240), the active-set method of
// src/sqp.rs:112-250 with N = 2 written out on scalars (GMW81 LDL^T of
// src/cholesky.rs:6-65 for one or two free variables).  One thread.
__device__ __forceinline__ int cls_self_qp(double q00, double q01, double q10, double q11, double c0, double c1,
                                           const Tune& tq, double& y0, double& y1) {
    return qp_simplex2(q00, q01, q10, q11, c0, c1, 0.5, 0.5, tq, y0, y1);
}

// The CLS estimator's step after its one moment pass (src/coefficients.rs:
// 218-268): c = (the pair's summed likelihood rows, biallelic from the moments
// plus the tri- and tetra-allelic sums) / (-M), every pair using all M kept
// sites; the simplex QP on the cohort's Q from 1/9, or the
// two-variable QP on (Delta1, Delta7) from (1/2, 1/2) for a self pair, with the
// cohort's iteration limit; then the Brier score, the condition estimate at
// g = Q delta + c, and the row (iters = the QP's iteration count).
__device__ __forceinline__ void cls_finish(const WaveArgs& A, SlotState& S, int s, const double* mom_s, int lane,
                                  const HalfGrp& grp) {
    const CohortDev& co = A.cohorts[S.cohort];
    const double m = co.cls_m;
    double Sg = 0.0, Ht[9];
    if (lane < 9) {
        rebuild_row(mom_s, lane, Sg, Ht);
        // the pair's tri- and tetra-allelic rows: c2 + (c3 + c4)
        if (co.cls_cmulti) Sg += co.cls_cmulti[(S.k - co.pair_begin) * 9 + lane];
    }
    double c[9];
    gather9(grp, Sg / -m, c);
    double Qr[9];
#pragma unroll
    for (int j = 0; j < 9; j++) Qr[j] = lane < 9 ? co.cls_q[lane * 9 + j] : 0.0;
    Tune tq = A.tune;
    tq.qp_max_iter = co.max_iter > (uint64_t)INT_MAX ? INT_MAX : (int)co.max_iter;
    double delta[9];
    int iters;
    if (co.kind == COHORT_TRIANGLE && S.x == S.y) {
        double e0 = 0.0, e6 = 0.0;
        int it2 = 0;
        if (lane == 0)
            it2 = cls_self_qp(co.cls_q[0], co.cls_q[6], co.cls_q[6 * 9], co.cls_q[6 * 9 + 6], c[0], c[6], tq, e0, e6);
        e0 = __shfl_sync(grp.mask, e0, 0, 16);
        e6 = __shfl_sync(grp.mask, e6, 0, 16);
        iters = __shfl_sync(grp.mask, it2, 0, 16);
#pragma unroll
        for (int j = 0; j < 9; j++) delta[j] = 0.0;
        delta[0] = e0;
        delta[6] = e6;
    } else {
        double y0[9];
#pragma unroll
        for (int j = 0; j < 9; j++) y0[j] = 1.0 / 9.0;
        iters = qp_simplex_rows(grp, Qr, c, y0, tq, lane, delta);
    }
    double qd[9];
    gather9(grp, lane < 9 ? dot_fma(9, Qr, delta) : 0.0, qd);
    const double quad = dot_fma(9, delta, qd);
    const double lin = 2.0 * dot_fma(9, c, delta);
    const double brier = (quad + lin) + 1.0;
    double g[9];
#pragma unroll
    for (int j = 0; j < 9; j++) g[j] = qd[j] + c[j];
    const double cond = condition_rows(grp, delta, g, Qr, tq.sqp_conv_tol);
    finish_slot(A, S, s, delta, brier, (uint64_t)iters, cond, lane);
}

// Schedules the slot's next pass at S.xt (lane 0 has written xt).  A pass in
// FP64 on FP32 lists first goes back through the admit step for FP64 lists.
__device__ inline void schedule_pass(const WaveArgs& A, SlotState& S, int s, int kind, int ev, int lane,
                                     const HalfGrp& grp) {
    if (lane == 0) {
        S.ev = ev;
        set_coefficients(S, kind);
    }
    if (kind == PASS_FP64 && !S.lists64) {
        if (lane == 0) {
            S.status = SLOT_RESORT;
            A.free_next[atomicAdd(&A.wc_next->n_free, 1)] = s;
            atomicAdd(&A.wc_next->n_resort, 1);
        }
        return;
    }
    if (lane == 0) S.status = SLOT_PASS;
    grp.sync();
    enqueue_pass<16>(A.pass_next, A.tasks_next, A.task_cap, A.wc_next, s, S, lane, grp.mask, A.unit_elems);
}

// Two slots per warp, one per half-warp (the row-parallel solver needs nine
// lanes), four blocks of four warps per SM (at most 128 registers a thread):
// the solver is latency-bound, so warps count for more than the few spilled
// values.  `lane` below is the lane's index in its half.
extern "C" __global__ void __launch_bounds__(128, 4) wave_solve_kernel(WaveArgs A) {
    extern __shared__ __align__(16) char smem[];
    const int wib = threadIdx.x >> 5, half = (threadIdx.x >> 4) & 1;
    const int lane = threadIdx.x & 15;
    const HalfGrp grp{half ? 0xFFFF0000u : 0x0000FFFFu};
    const int i = (blockIdx.x * WAVE_WPB + wib) * 2 + half;
    if (A.clk->stop) return;   // a device loop past its last wave
    if (threadIdx.x == 0) atomicMin(&A.clk->start[2], global_ns());
    const PhaseEnd pe{&A.clk->end[2], (threadIdx.x & 31) == 0};
    if (i >= A.wc_cur->n_pass) return;
    const int s = A.pass_cur[i];
    SlotState& S = A.slots[s];
    char* wsm = smem + wib * WARP_SMEM;
    double* mom_s = reinterpret_cast<double*>(wsm) + half * 64;
    const Tune& tu = A.tune;
    // ---- sum the units' partials in unit order: lane owns moments lane,
    // lane + 16 and lane + 32 (45 = the objective); a moment's units are those
    // of its shape
    {
        int us[6];
#pragma unroll
        for (int k = 0; k < 6; k++) us[k] = S.ustart[k];
        const double* P0 = A.partial + (int64_t)s * A.max_units * UNIT_VALS;
        // moment m belongs to shape A (0..10), B1 (11..18), B2 (19..26), C (27..39) or D (40..44)
        auto shape_of = [](int m) { return m < 11 ? 0 : m < 19 ? 1 : m < 27 ? 2 : m < 40 ? 3 : 4; };
        auto sum_range = [&](int u0, int u1, int col) {
            double acc = 0.0;
#pragma unroll 4
            for (int u = u0; u < u1; u++) acc += P0[(int64_t)u * UNIT_VALS + col];
            return acc;
        };
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int m = lane + 16 * k;
            if (m < NMOM) {
                const int sh = shape_of(m);
                mom_s[m] = sum_range(us[sh], us[sh + 1], m - shape_goff(sh));
            } else if (m == NMOM) {
                mom_s[m] = sum_range(0, us[5], UNIT_VALS - 1);
            }
        }
    }
    grp.sync();
    const int kind = S.kind;
    if (kind == PASS_CLS || kind == PASS_CLS64) {
        if (lane == 0) S.gh++;
        cls_finish(A, S, s, mom_s, lane, grp);
        return;
    }
    const double n = (double)S.n;
    double corr = 0.0;
    if (kind != PASS_FP64) {
        // FP32 passes ran on the hi coefficients
        if (lane == 0) mom_s[NMOM + 1] = lo_correction(mom_s, S.c32);
        grp.sync();
        corr = mom_s[NMOM + 1];
    }
    // the pair's tri- and tetra-allelic sums (ML path), units in order: lane
    // r < 9 takes gradient r and Hessian row r, lane 9 the objective term
    double ml_obj = 0.0, ml_g = 0.0, ml_h[9];
#pragma unroll
    for (int j = 0; j < 9; j++) ml_h[j] = 0.0;
    if (A.ml_units > 0) {
        const int nml = (A.cohorts[S.cohort].ml_nk + A.ml_chunk - 1) / A.ml_chunk;
        const double* P = A.ml_partial + (int64_t)s * A.ml_units * ML_VALS;
        for (int u = 0; u < nml; u++) {
            const double* Pu = P + (int64_t)u * ML_VALS;
            if (lane < 9) {
                ml_g += Pu[lane];
#pragma unroll
                for (int j = 0; j < 9; j++) ml_h[j] += Pu[9 + upper9(lane, j)];
            } else if (lane == 9) {
                ml_obj += Pu[54];
            }
        }
        ml_obj = grp.bcast(ml_obj, 9);
    }
    const double obj = mom_s[NMOM];
    double ft;
    if (kind == PASS_FP64) ft = -(obj + ml_obj) / n;
    else if (kind == PASS_FP32_DIRECT) ft = -((obj * 0.69314718055994530942 + corr) + ml_obj) / n;
    else ft = S.f - (obj + ml_obj) / n;
    double gt[9], Ht[9];
    {
        double Sg = 0.0;
#pragma unroll
        for (int j = 0; j < 9; j++) Ht[j] = 0.0;
        if (lane < 9) {
            rebuild_row(mom_s, lane, Sg, Ht);
            Sg += ml_g;
#pragma unroll
            for (int j = 0; j < 9; j++) Ht[j] = (Ht[j] + ml_h[j]) / n;
        }
        gather9(grp, -Sg / n, gt);
    }
    grp.sync();
    if (lane == 0) {
        S.gh++;
        if (kind == PASS_FP64) S.f64p++;
        if (kind == PASS_FP32_DIFF) S.diffp++;
    }
    // ---- the accepted state after this evaluation
    double x[9], g[9], Hr[9], f;
    bool fp64 = S.fp64 != 0;
    uint64_t it = S.it;
    const int ev = S.ev;
    bool after_reeval = false;
    if (ev == EV_TRIAL) {
        const double tt = tu.bls_sufficient_decrease * S.gp;
        const bool accept = ft <= S.f + S.alpha * tt;
        const int bls = S.bls + 1;
        if (!(accept || bls == tu.bls_max_iter)) {
            const double alpha = S.alpha * tu.bls_step_size_reduce;
            double xn[9];
#pragma unroll
            for (int k = 0; k < 9; k++) xn[k] = S.xc[k] + alpha * S.p[k];
            normalise9(xn);
            const int nkind = fp64 ? PASS_FP64
                                   : (fabs(alpha * S.gp) < DIFF_BELOW ? PASS_FP32_DIFF : PASS_FP32_DIRECT);
            if (lane == 0) {
                S.bls = bls;
                S.alpha = alpha;
                for (int k = 0; k < 9; k++) S.xt[k] = xn[k];
            }
            schedule_pass(A, S, s, nkind, EV_TRIAL, lane, grp);
            return;
        }
        it = it + 1;
    } else if (ev == EV_REEVAL) {
        fp64 = true;
        after_reeval = true;
    }
#pragma unroll
    for (int k = 0; k < 9; k++) { x[k] = S.xt[k]; g[k] = gt[k]; Hr[k] = Ht[k]; }
    f = ft;
    // persist the accepted point
    if (lane == 0) {
        for (int k = 0; k < 9; k++) { S.xc[k] = x[k]; S.g[k] = g[k]; }
        S.f = f;
        S.it = it;
        S.fp64 = fp64 ? 1 : 0;
        if (after_reeval) S.escalated = 1;
    }
    if (lane < 9) {
#pragma unroll
        for (int k = 0; k < 9; k++) S.H[lane * 9 + k] = Hr[k];
    }
    const uint64_t max_iter = A.cohorts[S.cohort].max_iter;
    if (it >= max_iter) {
        finish_slot(A, S, s, x, f, max_iter, CUDART_NAN, lane);
        return;
    }
    // ---- KKT test (src/sqp.rs:95-109) and the FP32 -> FP64 recheck
    double resid;
    bool conv = kkt_ok(x, g, tu.sqp_conv_tol, &resid);
    if (!fp64 && !after_reeval && (conv || resid < 1e-6)) {
        const int near = S.near_count + (conv ? 0 : 1);
        if (lane == 0) S.near_count = near;
        const double cond = conv ? condition_rows(grp, x, g, Hr, tu.sqp_conv_tol) : 0.0;
        const bool recheck = conv ? !(cond <= COND_RECHECK) : (near >= 3);
        if (recheck) {
            // FP64 re-evaluation at the same point; the pair stays FP64 from here.
            if (lane == 0)
                for (int k = 0; k < 9; k++) S.xt[k] = x[k];
            schedule_pass(A, S, s, PASS_FP64, EV_REEVAL, lane, grp);
            return;
        }
        if (conv) {
            finish_slot(A, S, s, x, f, it, cond, lane);
            return;
        }
    }
    if (conv) {
        finish_slot(A, S, s, x, f, it, condition_rows(grp, x, g, Hr, tu.sqp_conv_tol), lane);
        return;
    }
    // ---- QP step (src/sqp.rs:78-83): c = g - H x, y = QP(H, c, x).  Its
    // inputs go to the slot's QP buffer and the slot to this wave's QP list:
    // wave_qp_kernel solves them a thread per slot, wave_step_kernel takes the
    // step from the solution.
    double* Qb = A.qp_buf + (int64_t)s * QP_VALS;
    if (lane < 9) {
#pragma unroll
        for (int k = 0; k < 9; k++) Qb[lane * 9 + k] = Hr[k];
        Qb[81 + lane] = pick9(g, lane) - dot_fma(9, Hr, x);
    }
    if (lane == 0) A.qp_list[atomicAdd(&A.wc_cur->n_qp, 1)] = s;
}

// The QP of every slot in this wave's QP list, a thread per slot (kg_qp1.cuh,
// the same arithmetic as the row-parallel form); the solution replaces c's
// neighbour in the slot's QP buffer.  Three blocks per SM (168 registers, a
// few spilled) beat two without spills: the kernel is bound by its FP64
// dependency chains, so warps count more than registers.
extern "C" __global__ void __launch_bounds__(128, 3) wave_qp_kernel(WaveArgs A) {
    if (A.clk->stop) return;   // a device loop past its last wave
    const PhaseEnd pe{&A.clk->end[2], (threadIdx.x & 31) == 0};   // timed as part of the solve phase
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.wc_cur->n_qp) return;
    const int s = A.qp_list[i];
    double* Qb = A.qp_buf + (int64_t)s * QP_VALS;
    double c[9], x[9], y[9];
#pragma unroll
    for (int r = 0; r < 9; r++) {
        c[r] = Qb[81 + r];
        x[r] = A.slots[s].xc[r];
    }
    qp_simplex_thread(reinterpret_cast<const double (*)[9]>(Qb), c, x, A.tune, y);
#pragma unroll
    for (int k = 0; k < 9; k++) Qb[90 + k] = y[k];
}

// The step after each QP (src/sqp.rs:78-90): p = y - x, the first trial point
// x + p (normalised) and its pass.  Half-warp per slot, as the solve kernel.
extern "C" __global__ void __launch_bounds__(128) wave_step_kernel(WaveArgs A) {
    const int wib = threadIdx.x >> 5, half = (threadIdx.x >> 4) & 1;
    const int lane = threadIdx.x & 15;
    const HalfGrp grp{half ? 0xFFFF0000u : 0x0000FFFFu};
    const int i = (blockIdx.x * WAVE_WPB + wib) * 2 + half;
    if (A.clk->stop) return;   // a device loop past its last wave
    const PhaseEnd pe{&A.clk->end[2], (threadIdx.x & 31) == 0};
    if (i >= A.wc_cur->n_qp) return;
    const int s = A.qp_list[i];
    SlotState& S = A.slots[s];
    const double* Qb = A.qp_buf + (int64_t)s * QP_VALS;
    double x[9], g[9], p[9];
#pragma unroll
    for (int k = 0; k < 9; k++) {
        x[k] = S.xc[k];
        g[k] = S.g[k];
        p[k] = Qb[90 + k] - x[k];
    }
    const double gp = dot_fma(9, g, p);
    double xn[9];
#pragma unroll
    for (int k = 0; k < 9; k++) xn[k] = x[k] + 1.0 * p[k];
    normalise9(xn);
    const bool fp64 = S.fp64 != 0;
    const int nkind = fp64 ? PASS_FP64 : (fabs(gp) < DIFF_BELOW ? PASS_FP32_DIFF : PASS_FP32_DIRECT);
    grp.sync();   // every lane has read S before lane 0 writes it
    if (lane == 0) {
        for (int k = 0; k < 9; k++) { S.p[k] = p[k]; S.xt[k] = xn[k]; }
        S.gp = gp;
        S.alpha = 1.0;
        S.bls = 0;
    }
    schedule_pass(A, S, s, nkind, EV_TRIAL, lane, grp);
}

// ------------------------------------------------------------------- host

// The first wave's free list: every slot, and its count.
__global__ void wave_iota_kernel(int* v, int n, int* n_free) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
    if (i == 0) *n_free = n;
}

// The device loop's step after each wave: adds the wave's phase times and
// readies the next wave's counters (the next wave reads this wave's next
// counts as its current ones and accumulates into this wave's current ones).
// The loop stops once nothing is left (no pass and no resort scheduled, the
// queue exhausted) or after max_waves waves; the body's last step hands that
// to the loop condition.  A wave slot past the stop ran nothing and changes
// nothing.
__global__ void wave_end_kernel(WaveArgs A, int last, cudaGraphConditionalHandle loop,
                                unsigned long long max_waves) {
    if (threadIdx.x != 0) return;
    WaveClock* c = A.clk;
    if (!c->stop) {
        for (int i = 0; i < 3; i++)
            if (c->end[i] > c->start[i]) c->acc[i] += c->end[i] - c->start[i];
        c->waves++;
        const WaveCounts& n = *A.wc_next;
        if (n.n_pass == 0 && n.n_resort == 0 && *A.queue >= (unsigned long long)A.live->total_pairs) {
            c->stop = 1;
        } else if (c->waves >= max_waves) {
            c->stop = 1;
            c->limit_hit = 1;
        }
        *A.admit_task = 0;
        *A.pass_task = 0;
        *A.wc_cur = WaveCounts{};
    }
    for (int i = 0; i < 3; i++) {
        c->start[i] = ~0ull;
        c->end[i] = 0ull;
    }
    if (last) {
        c->iters++;
        cudaGraphSetConditional(loop, c->stop ? 0u : 1u);
    }
}

// ------------------------------------------------------------ the engine

struct WaveEngine::Impl {
    Workspace* ws = nullptr;
    cudaStream_t st = nullptr;
    RunConfig cfg;
    int64_t n_slots = 0, list_cap = 0, task_cap = 0;
    int max_units = 0, max_jobs = 0;
    int pass_blocks = 0, admit_blocks = 0, solve_blocks = 0, multi_blocks = 0, qp_blocks = 0;
    WaveArgs A{};
    WaveCounts* wc = nullptr;
    int* admit_task = nullptr;
    unsigned long long* q = nullptr;
    LiveQueue* live_d = nullptr;
    // host side
    std::vector<CohortDev> table;
    std::vector<char> reported;
    LiveQueue* live_h = nullptr;          // page-locked staging of the live extent
    WaveCounts* h_wc = nullptr;
    unsigned long long* h_q = nullptr;
    unsigned long long* h_done = nullptr;
    unsigned long long last_q = 0;
    int cur = 0;
    bool idle = true;
    uint64_t waves = 0, launches = 0;
    double phase[3] = {0.0, 0.0, 0.0}, total = 0.0;
    // one wave captured per parity of the current/next lists
    cudaGraph_t g[2] = {nullptr, nullptr};
    cudaGraphExec_t x[2] = {nullptr, nullptr};
    cudaEvent_t ev[2][4] = {};
    WaveArgs args[2]{};
    // the device loop: a WHILE node over two waves (first parity loop_first)
    WaveClock* clk = nullptr;
    WaveClock* clk_h = nullptr;
    cudaGraph_t lg = nullptr;
    cudaGraphExec_t lx = nullptr;
    int loop_first = -1;
    unsigned long long loop_cap = 0;
    // what open() was last called with, and the buffers its graphs point into
    bool opened = false;
    int64_t key_list_cap = 0, key_want = 0, key_expected = 0;
    int key_max_jobs = 0, key_precision = 0, key_bps = 0, key_dev = -1, key_ml_units = 0, key_ml_chunk = 0,
        key_unit = 0,
        key_divisor = 0;
    uint64_t key_iterations = 0;
    cudaStream_t key_st = nullptr;
    std::vector<void*> key_bufs;
    void drop_loop() {
        if (lx) cudaGraphExecDestroy(lx);
        if (lg) cudaGraphDestroy(lg);
        lx = nullptr;
        lg = nullptr;
        loop_first = -1;
    }
    ~Impl() {
        drop_loop();
        for (int p = 0; p < 2; p++) {
            if (x[p]) cudaGraphExecDestroy(x[p]);
            if (g[p]) cudaGraphDestroy(g[p]);
            for (auto& e : ev[p])
                if (e) cudaEventDestroy(e);
        }
    }
};

WaveEngine::WaveEngine() : d_(new Impl) {}
WaveEngine::~WaveEngine() { delete d_; }

int WaveEngine::open(Workspace& ws, cudaStream_t st, const RunConfig& cfg, int64_t list_cap,
                     int64_t expected_pairs, int max_jobs, std::string& err) {
    Impl& E = *d_;
    // list offsets travel as 32-bit values (tasks and the admit scatter)
    if (list_cap >= ((int64_t)1 << 31)) {
        err = "a pair's site lists would exceed 2^31 entries";
        return KG_EINVAL;
    }
    E.ws = &ws;
    E.st = st;
    E.cfg = cfg;
    E.list_cap = list_cap;
    E.max_jobs = std::max(1, max_jobs);
    int dev = 0;
    KG_WAVE_TRY(cudaGetDevice(&dev));
    if (ws.sm_count == 0) KG_WAVE_TRY(cudaDeviceGetAttribute(&ws.sm_count, cudaDevAttrMultiProcessorCount, dev));
    const bool same_call = E.opened && E.key_list_cap == list_cap && E.key_want == cfg.slots &&
                           E.key_expected == expected_pairs && E.key_max_jobs == E.max_jobs &&
                           E.key_precision == cfg.precision && E.key_bps == cfg.pass_blocks_per_sm &&
                           E.key_iterations == cfg.iterations && E.key_dev == dev && E.key_st == st &&
                           E.key_ml_units == cfg.ml_units && E.key_ml_chunk == cfg.ml_chunk &&
                           E.key_unit == cfg.unit_elems &&
                           E.key_divisor == cfg.slot_divisor;
    // work units: per shape at most ceil(list_cap / unit), over the five
    // shapes at most that + 5
    const int unit = cfg.unit_elems > 0 ? cfg.unit_elems : UNIT_ELEMS;
    const int64_t shape_units = (list_cap + unit - 1) / unit;
    E.max_units = (int)shape_units + 5;
    // slots: as many as the work and the memory allow
    const size_t per_slot = sizeof(double) * (size_t)list_cap + sizeof(double) * E.max_units * UNIT_VALS +
                            sizeof(SlotState) + 4 * sizeof(int) + 2 * 5 * shape_units * sizeof(int4);
    size_t fr = 0, tot = 0;
    // by default a fifth of the job's pairs, between 4,096 and 131,072: enough
    // to fill the waves, few enough that the last waves drain quickly
    const int64_t want = cfg.slots > 0 ? cfg.slots
                                       : std::min<int64_t>(131072, std::max<int64_t>(
                                                                      4096, expected_pairs / std::max(1, cfg.slot_divisor)));
    if (!same_call) {
        KG_WAVE_TRY(cudaMemGetInfo(&fr, &tot));
        const int64_t by_mem = (int64_t)((fr / 2) / per_slot);
        E.n_slots = std::max<int64_t>(1, std::min<int64_t>({want, by_mem, std::max<int64_t>(1, expected_pairs)}));
    }
    const int64_t n_slots = E.n_slots;
    E.task_cap = n_slots * shape_units;
    // device buffers (grown and reused through the workspace)
    KG_WAVE_TRY((cudaError_t)ws.scratch.reserve(sizeof(double) * (size_t)list_cap * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.partial.reserve(sizeof(double) * (size_t)E.max_units * UNIT_VALS * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.ml_partial.reserve(sizeof(double) * (size_t)std::max(1, cfg.ml_units) * ML_VALS *
                                                   (size_t)(cfg.ml_units > 0 ? n_slots : 1)));
    KG_WAVE_TRY((cudaError_t)ws.slots.reserve(sizeof(SlotState) * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.qp.reserve((sizeof(double) * QP_VALS + sizeof(int)) * (size_t)n_slots));
    KG_WAVE_TRY((cudaError_t)ws.lists_a.reserve(sizeof(int) * 2 * n_slots));   // pass lists
    KG_WAVE_TRY((cudaError_t)ws.lists_b.reserve(sizeof(int) * 2 * n_slots));   // free lists
    KG_WAVE_TRY((cudaError_t)ws.tasks.reserve(sizeof(int4) * 2 * 5 * E.task_cap));
    const size_t clk_off = (sizeof(WaveCounts) * 2 + 64 + sizeof(LiveQueue) + 15) & ~(size_t)15;
    KG_WAVE_TRY((cudaError_t)ws.counts.reserve(clk_off + sizeof(WaveClock)));
    KG_WAVE_TRY((cudaError_t)ws.queue.reserve(sizeof(unsigned long long) * 2));
    KG_WAVE_TRY((cudaError_t)ws.counters.reserve(sizeof(RunCounters)));
    KG_WAVE_TRY((cudaError_t)ws.table.reserve(sizeof(CohortDev) * E.max_jobs));
    KG_WAVE_TRY((cudaError_t)ws.done.reserve(sizeof(unsigned long long) * E.max_jobs));
    E.wc = reinterpret_cast<WaveCounts*>(ws.counts.p);
    E.admit_task = reinterpret_cast<int*>(E.wc + 2);
    E.live_d = reinterpret_cast<LiveQueue*>(reinterpret_cast<char*>(ws.counts.p) + sizeof(WaveCounts) * 2 + 64);
    E.clk = reinterpret_cast<WaveClock*>(reinterpret_cast<char*>(ws.counts.p) + clk_off);
    E.q = ws.queue.as<unsigned long long>();   // [0] pairs, [1] pass units
    int* pass_l[2] = {ws.lists_a.as<int>(), ws.lists_a.as<int>() + n_slots};
    int* free_l[2] = {ws.lists_b.as<int>(), ws.lists_b.as<int>() + n_slots};
    int4* tasks_l[2] = {ws.tasks.as<int4>(), ws.tasks.as<int4>() + 5 * E.task_cap};
    // host read-back (page-locked so the graph can copy into it)
    const size_t hbytes = sizeof(WaveClock) + sizeof(LiveQueue) + sizeof(WaveCounts) +
                          sizeof(unsigned long long) * (1 + E.max_jobs);
    KG_WAVE_TRY((cudaError_t)ws.host.reserve(hbytes));
    E.clk_h = ws.host.as<WaveClock>();
    E.live_h = reinterpret_cast<LiveQueue*>(E.clk_h + 1);
    E.h_wc = reinterpret_cast<WaveCounts*>(E.live_h + 1);
    E.h_q = reinterpret_cast<unsigned long long*>(E.h_wc + 1);
    E.h_done = E.h_q + 1;
    E.live_h->total_pairs = 0;
    E.live_h->n_cohorts = 0;
    const std::vector<void*> bufs{ws.scratch.p, ws.partial.p, ws.slots.p,    ws.lists_a.p, ws.lists_b.p,
                                  ws.tasks.p,   ws.counts.p,  ws.queue.p,    ws.counters.p, ws.table.p,
                                  ws.done.p,    ws.host.p,    ws.ml_partial.p, ws.qp.p};
    const bool reuse = same_call && bufs == E.key_bufs;
    // the job state of a fresh engine
    E.table.clear();
    E.reported.clear();
    E.last_q = 0;
    E.cur = 0;
    E.idle = true;
    E.waves = 0;
    for (double& ph : E.phase) ph = 0.0;
    E.total = 0.0;
    KG_WAVE_TRY(cudaMemsetAsync(ws.slots.p, 0, sizeof(SlotState) * n_slots, st));   // all SLOT_FREE
    KG_WAVE_TRY(cudaMemsetAsync(ws.queue.p, 0, sizeof(unsigned long long) * 2, st));
    KG_WAVE_TRY(cudaMemsetAsync(ws.counts.p, 0, clk_off + sizeof(WaveClock), st));
    KG_WAVE_TRY(cudaMemsetAsync(ws.counters.p, 0, sizeof(RunCounters), st));
    KG_WAVE_TRY(cudaMemsetAsync(ws.done.p, 0, sizeof(unsigned long long) * E.max_jobs, st));
    // the first wave's free list holds every slot
    wave_iota_kernel<<<(int)((n_slots + 255) / 256), 256, 0, st>>>(free_l[0], (int)n_slots, &E.wc[0].n_free);
    KG_WAVE_TRY(cudaGetLastError());
    if (reuse) {
        E.launches = 1;
        return KG_OK;
    }
    // per device, and cheap: set on every open (serving workers open engines
    // on several threads)
    KG_WAVE_TRY(
        cudaFuncSetAttribute(wave_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * PASS_WARP_SMEM));
    KG_WAVE_TRY(cudaFuncSetAttribute(wave_admit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     ADMIT_WARPS * ADMIT_WARP_SMEM));
    int occ = 0;
    KG_WAVE_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wave_pass_kernel, 128, 4 * PASS_WARP_SMEM));
    if (occ <= 0) {
        err = "site-pass kernel cannot be resident";
        return KG_ECUDA;
    }
    if (cfg.pass_blocks_per_sm > 0) occ = std::min(occ, cfg.pass_blocks_per_sm);
    E.pass_blocks = ws.sm_count * occ;
    int aocc = 0;
    KG_WAVE_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&aocc, wave_admit_kernel, ADMIT_WARPS * 32,
                                                              ADMIT_WARPS * ADMIT_WARP_SMEM));
    if (aocc <= 0) {
        err = "admit kernel cannot be resident";
        return KG_ECUDA;
    }
    E.admit_blocks = ws.sm_count * aocc;
    E.solve_blocks = (int)((n_slots + 2 * WAVE_WPB - 1) / (2 * WAVE_WPB));   // two slots per warp
    E.qp_blocks = (int)((n_slots + 127) / 128);                               // a thread per slot
    E.multi_blocks = 0;
    if (cfg.ml_units > 0) {
        int mocc = 0;
        KG_WAVE_TRY(cudaFuncSetAttribute(wave_multi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MULTI_SMEM));
        KG_WAVE_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&mocc, wave_multi_kernel, MULTI_WARPS * 32,
                                                                  MULTI_SMEM));
        E.multi_blocks = ws.sm_count * std::max(1, mocc);
    }
    WaveArgs& A = E.A;
    A.cohorts = ws.table.as<CohortDev>();
    A.live = E.live_d;
    A.precision = cfg.precision;
    A.queue = E.q;
    A.slots = ws.slots.as<SlotState>();
    A.n_slots = (int)n_slots;
    A.lists = ws.scratch.as<double>();
    A.list_stride = list_cap;
    A.partial = ws.partial.as<double>();
    A.max_units = E.max_units;
    A.task_cap = E.task_cap;
    A.pass_task = E.q + 1;
    A.admit_task = E.admit_task;
    A.tune = make_tune(cfg.iterations);
    A.counters = ws.counters.as<RunCounters>();
    A.cohort_done = ws.done.as<unsigned long long>();
    A.clk = E.clk;
    A.ml_partial = ws.ml_partial.as<double>();
    A.ml_units = cfg.ml_units;
    A.ml_chunk = cfg.ml_chunk;
    A.qp_buf = ws.qp.as<double>();
    A.qp_list = reinterpret_cast<int*>(A.qp_buf + (size_t)QP_VALS * n_slots);
    A.unit_elems = unit;
    E.drop_loop();
    // One wave (counter resets, admit, pass, solve, read-back) captured as a
    // CUDA graph per parity of the current/next lists, then replayed: one
    // launch per wave instead of a dozen API calls.  External event nodes time
    // its phases.
    const size_t wsm = WAVE_WPB * WARP_SMEM;
    WaveCounts* wc = E.wc;
    E.opened = false;
    for (int par = 0; par < 2; par++) {
        // graphs and events of an earlier open() with other sizes
        if (E.x[par]) cudaGraphExecDestroy(E.x[par]);
        if (E.g[par]) cudaGraphDestroy(E.g[par]);
        E.x[par] = nullptr;
        E.g[par] = nullptr;
        for (auto& e : E.ev[par]) {
            if (e) cudaEventDestroy(e);
            e = nullptr;
        }
    }
    for (int par = 0; par < 2; par++) {
        for (auto& e : E.ev[par]) KG_WAVE_TRY(cudaEventCreate(&e));
        const int cur = par, nxt = par ^ 1;
        WaveArgs Aw = A;
        Aw.pass_cur = pass_l[cur];
        Aw.pass_next = pass_l[nxt];
        Aw.free_cur = free_l[cur];
        Aw.free_next = free_l[nxt];
        Aw.tasks_cur = tasks_l[cur];
        Aw.tasks_next = tasks_l[nxt];
        Aw.wc_cur = wc + cur;
        Aw.wc_next = wc + nxt;
        E.args[par] = Aw;
        KG_WAVE_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        cudaError_t ce = cudaEventRecordWithFlags(E.ev[par][0], st, cudaEventRecordExternal);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(E.admit_task, 0, sizeof(int), st);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(E.q + 1, 0, sizeof(unsigned long long), st);
        if (ce == cudaSuccess) ce = cudaMemsetAsync(wc + nxt, 0, sizeof(WaveCounts), st);
        if (ce == cudaSuccess) {
            wave_admit_kernel<<<E.admit_blocks, ADMIT_WARPS * 32, ADMIT_WARPS * ADMIT_WARP_SMEM, st>>>(Aw);
            ce = cudaEventRecordWithFlags(E.ev[par][1], st, cudaEventRecordExternal);
        }
        if (ce == cudaSuccess) {
            wave_pass_kernel<<<E.pass_blocks, 128, WAVE_WPB * PASS_WARP_SMEM, st>>>(Aw);
            if (E.multi_blocks) wave_multi_kernel<<<E.multi_blocks, MULTI_WARPS * 32, MULTI_SMEM, st>>>(Aw);
            ce = cudaEventRecordWithFlags(E.ev[par][2], st, cudaEventRecordExternal);
        }
        if (ce == cudaSuccess) {
            wave_solve_kernel<<<E.solve_blocks, 128, wsm, st>>>(Aw);
            wave_qp_kernel<<<E.qp_blocks, 128, 0, st>>>(Aw);
            wave_step_kernel<<<E.solve_blocks, 128, 0, st>>>(Aw);
            ce = cudaEventRecordWithFlags(E.ev[par][3], st, cudaEventRecordExternal);
        }
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(E.h_wc, wc + nxt, sizeof(WaveCounts), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(E.h_q, E.q, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(E.h_done, A.cohort_done, sizeof(unsigned long long) * E.max_jobs,
                                 cudaMemcpyDeviceToHost, st);
        const cudaError_t ee = cudaStreamEndCapture(st, &E.g[par]);
        KG_WAVE_TRY(ce);
        KG_WAVE_TRY(ee);
        KG_WAVE_TRY(cudaGraphInstantiate(&E.x[par], E.g[par], 0));
    }
    E.launches = 1;
    E.opened = true;
    E.key_list_cap = list_cap;
    E.key_want = cfg.slots;
    E.key_expected = expected_pairs;
    E.key_max_jobs = E.max_jobs;
    E.key_precision = cfg.precision;
    E.key_bps = cfg.pass_blocks_per_sm;
    E.key_iterations = cfg.iterations;
    E.key_dev = dev;
    E.key_st = st;
    E.key_ml_units = cfg.ml_units;
    E.key_ml_chunk = cfg.ml_chunk;
    E.key_unit = cfg.unit_elems;
    E.key_divisor = cfg.slot_divisor;
    E.key_bufs = bufs;
    return KG_OK;
}

int WaveEngine::add(const std::vector<CohortDev>& jobs, std::string& err) {
    Impl& E = *d_;
    const cudaStream_t st = E.st;
    if ((int64_t)E.table.size() + (int64_t)jobs.size() > E.max_jobs) {
        err = "job table full";
        return KG_ENOMEM;
    }
    int64_t total = E.live_h->total_pairs;
    // claims past the old end (slots that found no pair) handed out no pair:
    // the queue restarts at the old end
    if (E.last_q > (unsigned long long)total) {
        const unsigned long long t = (unsigned long long)total;
        KG_WAVE_TRY(cudaMemcpyAsync(E.q, &t, sizeof(t), cudaMemcpyHostToDevice, st));
        KG_WAVE_TRY(cudaStreamSynchronize(st));   // t lives on this stack frame
        E.last_q = t;
    }
    const size_t first = E.table.size();
    for (CohortDev d : jobs) {
        d.pair_begin = total;
        if (d.max_iter == 0) d.max_iter = E.cfg.iterations;
        total += d.n_pairs;
        E.table.push_back(d);
        E.reported.push_back(0);
    }
    if (jobs.empty()) return KG_OK;
    KG_WAVE_TRY(cudaMemcpyAsync(const_cast<CohortDev*>(E.A.cohorts) + first, E.table.data() + first, sizeof(CohortDev) * jobs.size(),
                                cudaMemcpyHostToDevice, st));
    E.live_h->total_pairs = total;
    E.live_h->n_cohorts = (int32_t)E.table.size();
    KG_WAVE_TRY(cudaMemcpyAsync(E.live_d, E.live_h, sizeof(LiveQueue), cudaMemcpyHostToDevice, st));
    KG_WAVE_TRY(cudaStreamSynchronize(st));   // the staging is reused by the next add
    E.idle = false;
    return KG_OK;
}

int WaveEngine::wave(std::vector<int>& finished, std::string& err) {
    Impl& E = *d_;
    const cudaStream_t st = E.st;
    KG_WAVE_TRY(cudaGraphLaunch(E.x[E.cur], st));
    KG_WAVE_TRY(cudaStreamSynchronize(st));
    E.launches += E.multi_blocks ? 6 : 5;
    E.waves++;
    for (size_t k = 0; k < E.table.size(); k++)
        if (!E.reported[k] && E.h_done[k] >= (unsigned long long)E.table[k].n_pairs) {
            E.reported[k] = 1;
            finished.push_back((int)k);
        }
    for (int i = 0; i < 3; i++) {
        float ms = 0.f;
        KG_WAVE_TRY(cudaEventElapsedTime(&ms, E.ev[E.cur][i], E.ev[E.cur][i + 1]));
        E.phase[i] += ms;
        E.total += ms;
    }
    const WaveCounts h = *E.h_wc;
    E.last_q = *E.h_q;
    E.cur ^= 1;
    E.idle = (h.n_pass == 0 && h.n_resort == 0 && E.last_q >= (unsigned long long)E.live_h->total_pairs);
    return KG_OK;
}

int WaveEngine::run_until_idle(unsigned long long max_waves, std::string& err) {
    Impl& E = *d_;
    const cudaStream_t st = E.st;
    if (E.idle) return KG_OK;
    if (!E.lx || E.loop_first != E.cur || E.loop_cap != max_waves) {
        E.drop_loop();
        KG_WAVE_TRY(cudaGraphCreate(&E.lg, 0));
        cudaGraphConditionalHandle h;
        KG_WAVE_TRY(cudaGraphConditionalHandleCreate(&h, E.lg, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        KG_WAVE_TRY(cudaGraphAddNode(&node, E.lg, nullptr, 0, &np));
        cudaGraph_t body = np.conditional.phGraph_out[0];
        KG_WAVE_TRY(cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < 2; k++) {
            const WaveArgs& Aw = E.args[E.cur ^ k];
            wave_admit_kernel<<<E.admit_blocks, ADMIT_WARPS * 32, ADMIT_WARPS * ADMIT_WARP_SMEM, st>>>(Aw);
            wave_pass_kernel<<<E.pass_blocks, 128, WAVE_WPB * PASS_WARP_SMEM, st>>>(Aw);
            if (E.multi_blocks) wave_multi_kernel<<<E.multi_blocks, MULTI_WARPS * 32, MULTI_SMEM, st>>>(Aw);
            wave_solve_kernel<<<E.solve_blocks, 128, WAVE_WPB * WARP_SMEM, st>>>(Aw);
            wave_qp_kernel<<<E.qp_blocks, 128, 0, st>>>(Aw);
            wave_step_kernel<<<E.solve_blocks, 128, 0, st>>>(Aw);
            wave_end_kernel<<<1, 32, 0, st>>>(Aw, k, h, max_waves);
        }
        cudaGraph_t captured = nullptr;
        const cudaError_t ce = cudaGetLastError();
        const cudaError_t ee = cudaStreamEndCapture(st, &captured);
        KG_WAVE_TRY(ce);
        KG_WAVE_TRY(ee);
        KG_WAVE_TRY(cudaGraphInstantiate(&E.lx, E.lg, 0));
        E.loop_first = E.cur;
        E.loop_cap = max_waves;
    }
    // the first wave's counters (later waves: wave_end_kernel) and the clock
    KG_WAVE_TRY(cudaMemsetAsync(E.admit_task, 0, sizeof(int), st));
    KG_WAVE_TRY(cudaMemsetAsync(E.q + 1, 0, sizeof(unsigned long long), st));
    KG_WAVE_TRY(cudaMemsetAsync(E.wc + (E.cur ^ 1), 0, sizeof(WaveCounts), st));
    KG_WAVE_TRY(cudaMemsetAsync(E.clk, 0, sizeof(WaveClock), st));
    KG_WAVE_TRY(cudaMemsetAsync(E.clk->start, 0xFF, sizeof(E.clk->start), st));
    KG_WAVE_TRY(cudaGraphLaunch(E.lx, st));
    KG_WAVE_TRY(cudaMemcpyAsync(E.clk_h, E.clk, sizeof(WaveClock), cudaMemcpyDeviceToHost, st));
    KG_WAVE_TRY(cudaMemcpyAsync(E.h_q, E.q, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    KG_WAVE_TRY(cudaStreamSynchronize(st));
    const WaveClock c = *E.clk_h;
    for (int i = 0; i < 3; i++) {
        E.phase[i] += (double)c.acc[i] * 1e-6;
        E.total += (double)c.acc[i] * 1e-6;
    }
    E.waves += c.waves;
    E.launches += (E.multi_blocks ? 14 : 12) * c.iters;
    E.cur ^= (int)(c.waves & 1);
    E.last_q = *E.h_q;
    // the next wave's counts, as a host wave would have read them; the clock
    // no longer stops the kernels
    KG_WAVE_TRY(cudaMemcpyAsync(E.h_wc, E.wc + E.cur, sizeof(WaveCounts), cudaMemcpyDeviceToHost, st));
    KG_WAVE_TRY(cudaMemcpyAsync(E.h_done, E.A.cohort_done, sizeof(unsigned long long) * E.max_jobs,
                                cudaMemcpyDeviceToHost, st));
    KG_WAVE_TRY(cudaMemsetAsync(&E.clk->stop, 0, sizeof(unsigned int), st));
    KG_WAVE_TRY(cudaStreamSynchronize(st));
    const WaveCounts h = *E.h_wc;
    E.idle = (h.n_pass == 0 && h.n_resort == 0 && E.last_q >= (unsigned long long)E.live_h->total_pairs);
    for (size_t k = 0; k < E.table.size(); k++)
        if (E.h_done[k] >= (unsigned long long)E.table[k].n_pairs) E.reported[k] = 1;
    if (c.limit_hit) {
        err = "the device wave loop reached its wave limit";
        return KG_ETIMEOUT;
    }
    return KG_OK;
}

bool WaveEngine::idle() const { return d_->idle; }
int64_t WaveEngine::n_slots() const { return d_->n_slots; }
int64_t WaveEngine::list_cap() const { return d_->list_cap; }
int64_t WaveEngine::backlog() const {
    const int64_t total = d_->live_h ? d_->live_h->total_pairs : 0;
    return total - std::min<int64_t>(total, (int64_t)d_->last_q);
}

int WaveEngine::reset_jobs(std::string& err) {
    Impl& E = *d_;
    if (!E.idle) {
        err = "jobs still in flight";
        return KG_EINVAL;
    }
    E.table.clear();
    E.reported.clear();
    E.live_h->total_pairs = 0;
    E.live_h->n_cohorts = 0;
    E.last_q = 0;
    KG_WAVE_TRY(cudaMemcpyAsync(E.live_d, E.live_h, sizeof(LiveQueue), cudaMemcpyHostToDevice, E.st));
    KG_WAVE_TRY(cudaMemsetAsync(E.q, 0, sizeof(unsigned long long), E.st));
    KG_WAVE_TRY(cudaMemsetAsync(E.A.cohort_done, 0, sizeof(unsigned long long) * E.max_jobs, E.st));
    KG_WAVE_TRY(cudaStreamSynchronize(E.st));
    return KG_OK;
}

int WaveEngine::stats(kg_run_stats& stats, std::string& err) {
    Impl& E = *d_;
    RunCounters rc;
    KG_WAVE_TRY(cudaMemcpyAsync(&rc, E.ws->counters.p, sizeof(rc), cudaMemcpyDeviceToHost, E.st));
    KG_WAVE_TRY(cudaStreamSynchronize(E.st));
    stats.gh_passes = rc.gh_passes;
    stats.obj_passes = rc.obj_passes;
    stats.fp64_passes = rc.fp64_passes;
    stats.fp64_pairs = rc.fp64_pairs;
    stats.pair_sites = rc.pair_sites;
    stats.work_units = rc.work_units;
    stats.launches = E.launches;
    stats.flops_fp32 = rc.flops_fp32;
    stats.flops_fp64 = rc.flops_fp64;
    for (int k = 0; k < 5; k++) stats.shape_sites[k] = rc.shape_sites[k];
    stats.nonconverged = rc.nonconverged;
    stats.waves = E.waves;
    stats.slots = (uint64_t)E.n_slots;
    stats.admit_ms = E.phase[0];
    stats.pass_ms = E.phase[1];
    stats.solve_ms = E.phase[2];
    stats.pair_kernel_ms = E.total;
    if (rc.stalled_waits) {
        err = "a device wait for a list copy ran out of its limit";
        return KG_ETIMEOUT;
    }
    if (rc.nosite_pairs) {
        err = "a pair has no jointly observed segregating site (its row is NaN)";
        return KG_ENOSITES;
    }
    return KG_OK;
}

// All jobs of one call through one engine, waves until every pair is done.
int run_waves(const std::vector<PairJob>& jobs, const RunConfig& cfg_in, Workspace& ws,
              cudaStream_t st, kg_run_stats& stats, std::string& err,
              const std::vector<CohortDev>& table, int64_t total_pairs, int64_t list_cap) {
    (void)jobs;
    RunConfig cfg = cfg_in;
    int max_nk = 0;
    for (const CohortDev& d : table) max_nk = std::max(max_nk, (int)d.ml_nk);
    cfg.ml_units = (max_nk + ML_CHUNK - 1) / ML_CHUNK;
    cfg.ml_chunk = cfg.ml_units ? ((max_nk + cfg.ml_units - 1) / cfg.ml_units + 31) / 32 * 32 : 0;
    if (!ws.engine) ws.engine = std::make_shared<WaveEngine>();
    WaveEngine& eng = *ws.engine;
    int r = eng.open(ws, st, cfg, list_cap, total_pairs, (int)table.size(), err);
    if (r) return r;
    r = eng.add(table, err);
    if (r) return r;
    // KESTREL_HOST_WAVES=1 drives every wave from the host instead (kernel
    // profilers do not see kernels inside graphs with conditional nodes)
    const char* hw = std::getenv("KESTREL_HOST_WAVES");
    const bool host_waves = hw && hw[0] == '1';
    if (!cfg.job_done && !host_waves) {
        // the whole job in one graph launch: no host round trip per wave.
        // The wave limit only bounds a loop that would not end: a pair takes
        // at most (1 + backtracks) passes per iteration, twice over if it is
        // re-run in FP64, and a wave gives every slot one pass.
        const unsigned long long gens = (unsigned long long)(total_pairs / std::max<int64_t>(1, eng.n_slots())) + 2;
        uint64_t max_iter = cfg.iterations;
        for (const CohortDev& d : table) max_iter = std::max<uint64_t>(max_iter, (uint64_t)d.max_iter);
        const unsigned long long per_pair = 2ull * (max_iter + 2) * 16ull + 64ull;
        r = eng.run_until_idle(cfg.max_waves ? cfg.max_waves : gens * per_pair, err);
        if (r) return r;
        return eng.stats(stats, err);
    }
    std::vector<int> fin;
    uint64_t waves = 0;
    while (!eng.idle()) {
        if (cfg.max_waves && waves++ >= cfg.max_waves) {
            err = "the host wave loop reached its wave limit";
            return KG_ETIMEOUT;
        }
        fin.clear();
        r = eng.wave(fin, err);
        if (r) return r;
        if (cfg.job_done)
            for (int k : fin) cfg.job_done(k);
    }
    return eng.stats(stats, err);
}

}  // namespace kg
