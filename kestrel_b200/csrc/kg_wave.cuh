// kg_wave.cuh — the all-pairs estimator as waves over a batch of pair slots.
//
// A slot holds one pair's SQP state (src/sqp.rs:49-93) in HBM.  Each wave runs
// three small kernels, so each has the SM to itself with compact code:
//   admit : free slots take the next pairs from the device work queue (an atomic
//           counter over all cohorts' pairs) and build their shape lists;
//   pass  : a persistent kernel over work units (slot, shape, chunk of
//           unit_elems list entries, UNIT_ELEMS by default) streams the lists at
//           each slot's pending point and writes per-unit partial moments;
//   solve : one warp per slot sums its units' partials in a fixed order, rebuilds
//           f, g, H and advances the slot's SQP: KKT test, condition estimate,
//           simplex QP, Armijo line search.  Converged slots write their output
//           row and free the slot for the next admit.
// A pair's result depends only on its own lists and the fixed reduction order,
// never on which other pairs share its waves.
#pragma once

#include "kg_pair.cuh"

namespace kg {

constexpr int UNIT_ELEMS = 32768;  // list entries per pass work unit (the default; RunConfig::unit_elems)
constexpr int UNIT_VALS = 14;      // partial values per unit: <= 13 moments + objective

enum : int { SLOT_FREE = 0, SLOT_PASS = 1, SLOT_RESORT = 2 };
enum : int { EV_INIT = 0, EV_TRIAL = 1, EV_REEVAL = 2 };

struct SlotState {
    int64_t k;            // global work index of the pair
    int64_t x, y;
    int64_t start[5], cnt[5], n;
    int32_t ustart[6];    // prefix of work units over the five shapes
    int32_t cohort;
    int32_t status;       // SLOT_*
    int32_t lists64;      // the lists hold FP64 values
    int32_t fp64;         // passes run in FP64
    int32_t kind;         // PASS_* of the pending pass
    int32_t ev;           // EV_*: what the pending pass evaluates
    int32_t near_count;
    int32_t bls;
    int32_t escalated;
    int32_t gh, f64p, diffp;
    uint64_t it;
    double xc[9];         // accepted point
    double f;             // objective at xc
    double g[9];          // gradient at xc
    double H[81];         // Hessian at xc
    double p[9];          // search direction
    double gp;            // g . p
    double alpha;
    double xt[9];         // point of the pending pass
    Coef32 c32;           // its FP32 pass coefficients
    PassCoef c64;         // its FP64 pass coefficients
};

// Per-wave counters (one set for the current wave, one for the next).
struct WaveCounts {
    int n_pass;      // slots with a pending pass
    int n_free;      // slots for the admit step: free ones and those waiting for FP64 lists
    int n_resort;    // of those, slots waiting for FP64 lists
    int units[5];    // pass work units per shape, other than difference-objective ones (from each list's start)
    int n_qp;        // slots whose SQP step needs a QP (wave_qp_kernel) this wave
    int pad;
    int back[5];     // of the pass work units, difference-objective ones (from each list's end)
};

// The job table's extent, in device memory so that jobs can be appended
// between waves without touching the captured launches.
struct LiveQueue {
    int64_t total_pairs;   // pairs of all jobs so far (global work indices 0 .. total - 1)
    int32_t n_cohorts;     // jobs in the table
    int32_t pad;
};

// Device-side phase clock of the waves (%globaltimer, ns): each wave kernel
// lowers start[] as its blocks begin and raises end[] as its warps finish;
// wave_end_kernel adds end - start to acc[] and decides whether the device
// loop goes on.
struct WaveClock {
    unsigned long long start[3];   // admit, pass, solve of the current wave
    unsigned long long end[3];
    unsigned long long acc[3];     // summed over the waves of the device loop
    unsigned long long waves;      // waves the device loop ran
    unsigned long long iters;      // loop bodies (two wave slots each)
    unsigned int stop;             // set once the job is done or the limit is hit
    unsigned int limit_hit;
};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Raises the phase's end time as the scope closes (one thread per warp or
// block, as the kernel chooses).
struct PhaseEnd {
    unsigned long long* end;
    bool on;
    __device__ ~PhaseEnd() {
        if (on) atomicMax(end, global_ns());
    }
};

struct WaveArgs {
    const CohortDev* cohorts;
    const LiveQueue* live;
    int precision;
    unsigned long long* queue;     // next pair (global work index)
    SlotState* slots;
    int n_slots;
    double* lists;                 // per slot: list_stride 8-byte words
    int64_t list_stride;
    double* partial;               // per slot: max_units * UNIT_VALS
    int max_units;
    // the current wave's lists (filled by the previous solve step and this
    // wave's admit step) and the next wave's (filled by this solve step)
    int* pass_cur;
    int* pass_next;
    int* free_cur;
    int* free_next;
    int4* tasks_cur;               // per shape: task_cap entries (PassTask)
    int4* tasks_next;
    int64_t task_cap;
    WaveCounts* wc_cur;
    WaveCounts* wc_next;
    unsigned long long* pass_task; // pass work-unit counter
    int* admit_task;               // admit entry counter
    Tune tune;
    RunCounters* counters;
    unsigned long long* cohort_done;   // finished pairs per cohort
    WaveClock* clk;
    double* ml_partial;            // per slot: ml_units * ML_VALS sums of its tri-/tetra-allelic sites
    int ml_units;                  // their work units per slot (0: no cohort has such sites)
    int ml_chunk;                  // kept sites per such unit (a multiple of 32, at most ML_CHUNK)
    double* qp_buf;                // per slot QP_VALS: Q (9 x 9 row-major), c, the solution y
    int* qp_list;                  // the slots of this wave's QPs (wc_cur->n_qp of them)
    int unit_elems;                // list entries per pass work unit
};

// Work units of the ML path's tri- and tetra-allelic sites: at most ML_CHUNK
// kept sites each, the largest cohort's sites split evenly; per unit 9
// gradient sums, the 45 Hessian sums of the upper triangle (row-major) and the
// objective term.
constexpr int ML_CHUNK = 8192;
constexpr int ML_VALS = 56;
// a slot's QP: Q at 0, c at 81, the solution at 90
constexpr int QP_VALS = 100;

__device__ __forceinline__ int shape_ng(int s) { return s == 0 ? 4 : s == 3 ? 4 : s == 4 ? 2 : 3; }
__device__ __forceinline__ int shape_nh(int s) { return s == 0 ? 7 : s == 3 ? 9 : s == 4 ? 3 : 5; }
__device__ __forceinline__ int shape_goff(int s) { return s == 0 ? 0 : s == 1 ? 11 : s == 2 ? 19 : s == 3 ? 27 : 40; }

// Coefficients of the pending pass at xt (relative to the accepted xc for the
// log(d_new/d_old) objective).  Called by lane 0.
__device__ inline void set_coefficients(SlotState& S, int kind) {
    PassCoef k;
    make_coef(S.xt, k);
    S.c64 = k;
    Coef32 c;
    for (int i = 0; i < 4; i++) { c.a[i] = split(k.a[i]); c.c[i] = split(k.c[i]); }
    for (int i = 0; i < 3; i++) { c.b1[i] = split(k.b1[i]); c.b2[i] = split(k.b2[i]); }
    for (int i = 0; i < 2; i++) c.d[i] = split(k.d[i]);
    double s[9];
    for (int i = 0; i < 9; i++) s[i] = S.xt[i] - S.xc[i];
    PassCoef ks;
    make_coef(s, ks);
    for (int i = 0; i < 4; i++) { c.sa[i] = (float)ks.a[i]; c.sc[i] = (float)ks.c[i]; }
    for (int i = 0; i < 3; i++) { c.sb1[i] = (float)ks.b1[i]; c.sb2[i] = (float)ks.b2[i]; }
    for (int i = 0; i < 2; i++) c.sd[i] = (float)ks.d[i];
    S.c32 = c;
    S.kind = kind;
}

__device__ inline void units_from_counts(SlotState& S, int unit) {
    S.ustart[0] = 0;
    for (int s = 0; s < 5; s++) S.ustart[s + 1] = S.ustart[s] + (int)((S.cnt[s] + unit - 1) / unit);
}

__device__ __forceinline__ void decode_pair(const WaveArgs& A, int64_t k, int& c, int64_t& j,
                                            int64_t& x, int64_t& y) {
    // the last job whose range starts at or before k
    int lo = 0, hi = A.live->n_cohorts - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (A.cohorts[mid].pair_begin <= k) lo = mid;
        else hi = mid - 1;
    }
    c = lo;
    const CohortDev& co = A.cohorts[c];
    j = k - co.pair_begin;
    if (co.kind == COHORT_TRIANGLE) {
        double b = 2.0 * (double)co.n_x + 1.0;
        double disc = b * b - 8.0 * (double)j;
        int64_t xi = (int64_t)floor((b - sqrt(fmax(disc, 0.0))) * 0.5);
        const int64_t ns = co.n_x;
        if (xi < 0) xi = 0;
        if (xi > ns - 1) xi = ns - 1;
        auto off = [ns](int64_t r) { return r * ns - r * (r - 1) / 2; };
        while (xi > 0 && off(xi) > j) xi--;
        while (xi + 1 < ns && off(xi + 1) <= j) xi++;
        x = xi;
        y = xi + (j - off(xi));
    } else {
        x = j / co.n_y;
        y = j - x * co.n_y;
    }
}

// A pass work unit as stored in the task lists: everything the pass kernel
// needs before its first list copy, {slot, unit, list offset, length | kind << 24}.
__device__ __forceinline__ int4 make_task(int s, int u, int64_t off, int64_t len, int kind) {
    return make_int4(s, u, (int)off, (int)len | (kind << 24));
}

// Queues slot s for a pass in the wave whose lists are (pass, tasks, wc): its
// work units go to the shape-major task lists, so that the warps of the pass
// kernel run one shape's code at a time; within a shape's list, units of
// difference-objective passes fill it from the end and the others from the
// start, so the warps also run one pass kind's code at a time (mixing the two
// kinds took 2.5% more pass time).  Called after S.ustart is set by W
// lanes (a warp or a half-warp, given by mask); lane is the index among them.
template <int W>
__device__ inline void enqueue_pass(int* pass, int4* tasks, int64_t task_cap, WaveCounts* wc, int s,
                                    const SlotState& S, int lane, unsigned mask, int unit) {
#pragma unroll 1
    for (int sh = 0; sh < 5; sh++) {
        const int u0 = S.ustart[sh], nu = S.ustart[sh + 1] - u0;
        if (nu == 0) continue;
        const int kind = S.kind;
        const bool from_end = (kind == PASS_FP32_DIFF);
        int base = 0;
        if (lane == 0) base = atomicAdd(from_end ? &wc->back[sh] : &wc->units[sh], nu);
        base = __shfl_sync(mask, base, 0, W);
        const int64_t st = S.start[sh], cnt = S.cnt[sh];
        for (int i = lane; i < nu; i += W) {
            const int64_t c0 = (int64_t)i * unit;
            const int64_t at = from_end ? task_cap - 1 - (base + i) : base + i;
            tasks[sh * task_cap + at] = make_task(s, u0 + i, st + c0, min((int64_t)unit, cnt - c0), kind);
        }
    }
    if (lane == 0) pass[atomicAdd(&wc->n_pass, 1)] = s;
}

__device__ inline void write_row(kg_output* out, int64_t x, int64_t y, const double* d, double obj,
                                 uint64_t iters, double cond, int lane) {
    kg_output row;
    row.x = (uint64_t)x;
    row.y = (uint64_t)y;
    for (int i = 0; i < 9; i++) row.jacquard[i] = d[i];
    row.obj = obj;
    row.iters = iters;
    row.cond = cond;
    const uint64_t* src = reinterpret_cast<const uint64_t*>(&row);
    uint64_t wv = 0;
#pragma unroll
    for (int i = 0; i < 14; i++)
        if (lane == i) wv = src[i];
    if (lane < 14) reinterpret_cast<uint64_t*>(out)[lane] = wv;
}

}  // namespace kg
