// kg_wave.cu — wave kernels (admit / pass / solve) and their host loop.
// See kg_wave.cuh for the scheme; the SQP logic restates src/sqp.rs:49-310.
#include <algorithm>
#include <cstring>

#include "kg_engine.h"
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

extern "C" __global__ void __launch_bounds__(128) wave_admit_kernel(WaveArgs A, int* pass_list,
                                                                     int* n_pass) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int s = blockIdx.x * WAVE_WPB + wib;
    if (s >= A.n_slots) return;
    char* wsm = smem + wib * WARP_SMEM;
    SlotState& S = A.slots[s];
    void* lists = A.lists + (int64_t)s * A.list_stride;
    const int status = S.status;
    if (status == SLOT_RESORT) {
        PairLists pl;
        for (int i = 0; i < 5; i++) { pl.start[i] = S.start[i]; pl.cnt[i] = S.cnt[i]; }
        pl.n = S.n;
        scatter_shapes<double>(A.cohorts[S.cohort], S.x, S.y, lane, pl, static_cast<double*>(lists), wsm);
        __syncwarp();
        if (lane == 0) {
            S.lists64 = 1;
            S.status = SLOT_PASS;
            pass_list[atomicAdd(n_pass, 1)] = s;
        }
        return;
    }
    if (status != SLOT_FREE) return;
    for (;;) {
        unsigned long long k = 0;
        if (lane == 0) k = atomicAdd(A.queue, 1ull);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= (unsigned long long)A.total_pairs) return;
        int c;
        int64_t j, x, y;
        decode_pair(A, (int64_t)k, c, j, x, y);
        const CohortDev& co = A.cohorts[c];
        PairLists pl;
        count_shapes(co, x, y, lane, pl);
        if (pl.n == 0) {
            double nan9[9];
            for (int i = 0; i < 9; i++) nan9[i] = CUDART_NAN;
            write_row(co.out + j, x, y, nan9, CUDART_NAN, 0, CUDART_NAN, lane);
            if (lane == 0) atomicAdd(&A.counters->nosite_pairs, 1ull);
            continue;
        }
        const bool f64 = (A.precision == 1);
        if (f64) scatter_shapes<double>(co, x, y, lane, pl, static_cast<double*>(lists), wsm);
        else scatter_shapes<float>(co, x, y, lane, pl, static_cast<float*>(lists), wsm);
        __syncwarp();
        if (lane == 0) {
            S.k = (int64_t)k;
            S.x = x;
            S.y = y;
            S.cohort = c;
            for (int i = 0; i < 5; i++) { S.start[i] = pl.start[i]; S.cnt[i] = pl.cnt[i]; }
            S.n = pl.n;
            units_from_counts(S);
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
            set_coefficients(S, f64 ? PASS_FP64 : PASS_FP32_DIRECT);
            S.status = SLOT_PASS;
            pass_list[atomicAdd(n_pass, 1)] = s;
        }
        return;
    }
}

// ------------------------------------------------------------------- pass

template <int SH>
__device__ __forceinline__ void run_unit(const void* lists, bool l64, int64_t off, int64_t len,
                                         const void* kbuf, bool diff, int lane, LaneSums& ls) {
    if (l64)
        stream64<SH>(static_cast<const double*>(lists) + off, len, reinterpret_cast<const PassCoef*>(kbuf),
                     lane, ls);
    else
        stream32<SH>(static_cast<const float*>(lists) + off, len, reinterpret_cast<const Coef32*>(kbuf),
                     diff, lane, ls);
}

extern "C" __global__ void __launch_bounds__(128, 4) wave_pass_kernel(WaveArgs A) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    char* wsm = smem + wib * WARP_SMEM;
    char* kbuf = wsm + WARP_SMEM_BUF;
    const int np = *A.n_pass;
    const int64_t ntask = (int64_t)np * A.max_units;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(A.task, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if ((int64_t)t >= ntask) break;
        const int s = A.pass_list[t / A.max_units];
        const int u = (int)(t % A.max_units);
        const SlotState& S = A.slots[s];
        if (u >= S.ustart[5]) continue;
        int sh = 0;
        while (u >= S.ustart[sh + 1]) sh++;
        const int64_t c0 = (int64_t)(u - S.ustart[sh]) * UNIT_ELEMS;
        const int64_t off = S.start[sh] + c0;
        const int64_t len = min((int64_t)UNIT_ELEMS, S.cnt[sh] - c0);
        const int kind = S.kind;
        const bool l64 = (kind == PASS_FP64);
        // the pending pass's coefficients into this warp's shared memory
        const int nwords = l64 ? (int)(sizeof(PassCoef) / 4) : (int)(sizeof(Coef32) / 4);
        const uint32_t* src = l64 ? reinterpret_cast<const uint32_t*>(&S.c64)
                                  : reinterpret_cast<const uint32_t*>(&S.c32);
        for (int w = lane; w < nwords; w += 32) reinterpret_cast<uint32_t*>(kbuf)[w] = src[w];
        __syncwarp();
        const void* lists = A.lists + (int64_t)s * A.list_stride;
        const bool diff = (kind == PASS_FP32_DIFF);
        LaneSums ls;
        ls.obj = 0.0;
        switch (sh) {
        case 0: run_unit<0>(lists, l64, off, len, kbuf, diff, lane, ls); break;
        case 1: run_unit<1>(lists, l64, off, len, kbuf, diff, lane, ls); break;
        case 2: run_unit<2>(lists, l64, off, len, kbuf, diff, lane, ls); break;
        case 3: run_unit<3>(lists, l64, off, len, kbuf, diff, lane, ls); break;
        default: run_unit<4>(lists, l64, off, len, kbuf, diff, lane, ls); break;
        }
        const int go = shape_goff(sh), nv = shape_ng(sh) + shape_nh(sh);
        double* P = A.partial + ((int64_t)s * A.max_units + u) * UNIT_VALS;
        for (int i = 0; i < nv; i++) {
            const double v = warp_sum(ls.m[go + i]);
            if (lane == 0) P[i] = v;
        }
        const double ob = warp_sum(ls.obj);
        if (lane == 0) P[UNIT_VALS - 1] = ob;
        __syncwarp();
    }
}

// ------------------------------------------------------------------ solve

__device__ inline void finish_slot(const WaveArgs& A, SlotState& S, const double* x, double f,
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
        if (iters >= A.tune.sqp_max_iter) atomicAdd(&C->nonconverged, 1ull);
        const int p32 = S.gh - S.f64p;
        unsigned long long f32 = 0, f64 = 0;
        for (int s = 0; s < 5; s++) {
            atomicAdd(&C->shape_sites[s], (unsigned long long)S.cnt[s]);
            f32 += (unsigned long long)S.cnt[s] * (unsigned long long)(p32 * flops_direct(s) + S.diffp * flops_diff_extra(s));
            f64 += (unsigned long long)S.cnt[s] * (unsigned long long)(S.f64p * flops_direct(s));
        }
        atomicAdd(&C->flops_fp32, f32);
        atomicAdd(&C->flops_fp64, f64);
        S.status = SLOT_FREE;
    }
}

// Schedules the slot's next pass at S.xt (lane 0 has written xt).
__device__ inline void schedule_pass(const WaveArgs& A, SlotState& S, int s, int kind, int ev, int lane) {
    if (lane == 0) {
        S.ev = ev;
        set_coefficients(S, kind);
        if (kind == PASS_FP64 && !S.lists64) {
            S.status = SLOT_RESORT;
            atomicAdd(A.n_resort, 1);
        } else {
            S.status = SLOT_PASS;
            A.next_list[atomicAdd(A.n_next, 1)] = s;
        }
    }
}

extern "C" __global__ void __launch_bounds__(128) wave_solve_kernel(WaveArgs A) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int i = blockIdx.x * WAVE_WPB + wib;
    if (i >= *A.n_pass) return;
    const int s = A.pass_list[i];
    SlotState& S = A.slots[s];
    char* wsm = smem + wib * WARP_SMEM;
    double* mom_s = reinterpret_cast<double*>(wsm);
    const Tune& tu = A.tune;
    // ---- sum the units' partials in unit order: lane owns moments lane and lane + 32
    {
        double m0 = 0.0, m1 = 0.0;
        const int nu = S.ustart[5];
        const double* P0 = A.partial + (int64_t)s * A.max_units * UNIT_VALS;
        int sh = 0;
        for (int u = 0; u < nu; u++) {
            while (u >= S.ustart[sh + 1]) sh++;
            const double* P = P0 + (int64_t)u * UNIT_VALS;
            const int go = shape_goff(sh), nv = shape_ng(sh) + shape_nh(sh);
            if (lane >= go && lane < go + nv) m0 += P[lane - go];
            const int l1 = lane + 32;
            if (l1 == NMOM) m1 += P[UNIT_VALS - 1];
            else if (l1 < NMOM && l1 >= go && l1 < go + nv) m1 += P[l1 - go];
        }
        mom_s[lane] = m0;
        if (lane + 32 <= NMOM) mom_s[lane + 32] = m1;
    }
    __syncwarp();
    const int kind = S.kind;
    const double n = (double)S.n;
    const double obj = mom_s[NMOM];
    double ft;
    if (kind == PASS_FP64) ft = -obj / n;
    else if (kind == PASS_FP32_DIRECT) ft = -(obj * 0.69314718055994530942) / n;
    else ft = S.f - obj / n;
    double gt[9], Ht[9];
    {
        double Sg = 0.0;
#pragma unroll
        for (int j = 0; j < 9; j++) Ht[j] = 0.0;
        if (lane < 9) {
            rebuild_row(mom_s, lane, Sg, Ht);
#pragma unroll
            for (int j = 0; j < 9; j++) Ht[j] = Ht[j] / n;
        }
        gather9(-Sg / n, gt);
    }
    __syncwarp();
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
            schedule_pass(A, S, s, nkind, EV_TRIAL, lane);
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
    if (it >= tu.sqp_max_iter) {
        finish_slot(A, S, x, f, tu.sqp_max_iter, CUDART_NAN, lane);
        return;
    }
    // ---- KKT test (src/sqp.rs:95-109) and the FP32 -> FP64 recheck
    double resid;
    bool conv = kkt_ok(x, g, tu.sqp_conv_tol, &resid);
    if (!fp64 && !after_reeval && (conv || resid < 1e-6)) {
        const int near = S.near_count + (conv ? 0 : 1);
        if (lane == 0) S.near_count = near;
        const double cond = conv ? condition_rows(x, g, Hr, tu.sqp_conv_tol) : 0.0;
        const bool recheck = conv ? !(cond <= COND_RECHECK) : (near >= 3);
        if (recheck) {
            // FP64 re-evaluation at the same point; the pair stays FP64 from here.
            if (lane == 0)
                for (int k = 0; k < 9; k++) S.xt[k] = x[k];
            schedule_pass(A, S, s, PASS_FP64, EV_REEVAL, lane);
            return;
        }
        if (conv) {
            finish_slot(A, S, x, f, it, cond, lane);
            return;
        }
    }
    if (conv) {
        finish_slot(A, S, x, f, it, condition_rows(x, g, Hr, tu.sqp_conv_tol), lane);
        return;
    }
    // ---- QP step (src/sqp.rs:78-83): c = g - H x, y = QP(H, c, x), p = y - x
    double cr = 0.0;
    if (lane < 9) cr = pick9(g, lane) - dot_fma(9, Hr, x);
    double c[9], y[9], p[9];
    gather9(cr, c);
    qp_simplex_rows(Hr, c, x, tu, lane, y);
#pragma unroll
    for (int k = 0; k < 9; k++) p[k] = y[k] - x[k];
    const double gp = dot_fma(9, g, p);
    double xn[9];
#pragma unroll
    for (int k = 0; k < 9; k++) xn[k] = x[k] + 1.0 * p[k];
    normalise9(xn);
    const int nkind = fp64 ? PASS_FP64 : (fabs(gp) < DIFF_BELOW ? PASS_FP32_DIFF : PASS_FP32_DIRECT);
    if (lane == 0) {
        for (int k = 0; k < 9; k++) { S.p[k] = p[k]; S.xt[k] = xn[k]; }
        S.gp = gp;
        S.alpha = 1.0;
        S.bls = 0;
    }
    schedule_pass(A, S, s, nkind, EV_TRIAL, lane);
}

// ------------------------------------------------------------------- host

int run_waves(const std::vector<PairJob>& jobs, const RunConfig& cfg, Workspace& ws,
              cudaStream_t st, kg_run_stats& stats, std::string& err,
              const std::vector<CohortDev>& table, int64_t total_pairs, int64_t list_cap) {
    int dev = 0;
    KG_WAVE_TRY(cudaGetDevice(&dev));
    if (ws.sm_count == 0) KG_WAVE_TRY(cudaDeviceGetAttribute(&ws.sm_count, cudaDevAttrMultiProcessorCount, dev));
    // slots: as many as the work and the memory allow
    const int max_units = (int)((list_cap + UNIT_ELEMS - 1) / UNIT_ELEMS) + 5;
    const size_t per_slot = sizeof(double) * (size_t)list_cap + sizeof(double) * max_units * UNIT_VALS +
                            sizeof(SlotState) + 2 * sizeof(int);
    size_t fr = 0, tot = 0;
    KG_WAVE_TRY(cudaMemGetInfo(&fr, &tot));
    int64_t want = cfg.slots > 0 ? cfg.slots : 8192;
    int64_t by_mem = (int64_t)((fr / 2) / per_slot);
    int64_t n_slots = std::max<int64_t>(1, std::min<int64_t>({want, by_mem, total_pairs}));
    // device buffers (grown and reused through the workspace)
    KG_WAVE_TRY((cudaError_t)ws.scratch.reserve(sizeof(double) * (size_t)list_cap * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.partial.reserve(sizeof(double) * (size_t)max_units * UNIT_VALS * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.slots.reserve(sizeof(SlotState) * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.lists_a.reserve(sizeof(int) * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.lists_b.reserve(sizeof(int) * n_slots));
    KG_WAVE_TRY((cudaError_t)ws.counts.reserve(sizeof(int) * 8));
    KG_WAVE_TRY((cudaError_t)ws.queue.reserve(sizeof(unsigned long long) * 2));
    KG_WAVE_TRY((cudaError_t)ws.counters.reserve(sizeof(RunCounters)));
    KG_WAVE_TRY((cudaError_t)ws.table.reserve(sizeof(CohortDev) * table.size()));
    KG_WAVE_TRY(cudaMemcpyAsync(ws.table.p, table.data(), sizeof(CohortDev) * table.size(),
                                cudaMemcpyHostToDevice, st));
    KG_WAVE_TRY(cudaMemsetAsync(ws.slots.p, 0, sizeof(SlotState) * n_slots, st));   // all SLOT_FREE
    KG_WAVE_TRY(cudaMemsetAsync(ws.queue.p, 0, sizeof(unsigned long long) * 2, st));
    KG_WAVE_TRY(cudaMemsetAsync(ws.counts.p, 0, sizeof(int) * 8, st));
    KG_WAVE_TRY(cudaMemsetAsync(ws.counters.p, 0, sizeof(RunCounters), st));
    static bool attr = false;
    if (!attr) {
        KG_WAVE_TRY(cudaFuncSetAttribute(wave_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * WARP_SMEM));
        attr = true;
    }
    int occ = 0;
    KG_WAVE_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wave_pass_kernel, 128, 4 * WARP_SMEM));
    if (occ <= 0) {
        err = "site-pass kernel cannot be resident";
        return KG_ECUDA;
    }
    if (cfg.pass_blocks_per_sm > 0) occ = std::min(occ, cfg.pass_blocks_per_sm);
    const int pass_blocks = ws.sm_count * occ;
    int* counts = ws.counts.as<int>();   // [0] n_a, [1] n_b, [2] n_resort
    unsigned long long* q = ws.queue.as<unsigned long long>();   // [0] pairs, [1] pass units
    WaveArgs A;
    A.cohorts = ws.table.as<CohortDev>();
    A.n_cohorts = (int)table.size();
    A.precision = cfg.precision;
    A.total_pairs = total_pairs;
    A.queue = q;
    A.slots = ws.slots.as<SlotState>();
    A.n_slots = (int)n_slots;
    A.lists = ws.scratch.as<double>();
    A.list_stride = list_cap;
    A.partial = ws.partial.as<double>();
    A.max_units = max_units;
    A.n_resort = counts + 2;
    A.task = q + 1;
    A.tune = make_tune(cfg.iterations);
    A.counters = ws.counters.as<RunCounters>();
    int* lst[2] = {ws.lists_a.as<int>(), ws.lists_b.as<int>()};
    int cur = 0;
    const int slot_blocks = (int)((n_slots + WAVE_WPB - 1) / WAVE_WPB);
    const size_t wsm = WAVE_WPB * WARP_SMEM;
    // events: [0] start, then per wave admit / pass / solve ends
    cudaEvent_t ev[4];
    for (auto& e : ev) KG_WAVE_TRY(cudaEventCreate(&e));
    struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int i = 0; i < 4; i++) cudaEventDestroy(e[i]); } } eg{ev};
    uint64_t waves = 0, launches = 0;
    double phase[3] = {0.0, 0.0, 0.0}, total = 0.0;
    for (;;) {
        A.pass_list = lst[cur];
        A.n_pass = counts + cur;
        A.next_list = lst[cur ^ 1];
        A.n_next = counts + (cur ^ 1);
        KG_WAVE_TRY(cudaEventRecord(ev[0], st));
        wave_admit_kernel<<<slot_blocks, 128, wsm, st>>>(A, lst[cur], counts + cur);
        KG_WAVE_TRY(cudaMemsetAsync(q + 1, 0, sizeof(unsigned long long), st));
        KG_WAVE_TRY(cudaEventRecord(ev[1], st));
        wave_pass_kernel<<<pass_blocks, 128, wsm, st>>>(A);
        KG_WAVE_TRY(cudaEventRecord(ev[2], st));
        KG_WAVE_TRY(cudaMemsetAsync(counts + (cur ^ 1), 0, sizeof(int), st));
        KG_WAVE_TRY(cudaMemsetAsync(counts + 2, 0, sizeof(int), st));
        wave_solve_kernel<<<slot_blocks, 128, wsm, st>>>(A);
        KG_WAVE_TRY(cudaGetLastError());
        KG_WAVE_TRY(cudaEventRecord(ev[3], st));
        launches += 3;
        waves++;
        int h[3];
        unsigned long long hq = 0;
        KG_WAVE_TRY(cudaMemcpyAsync(h, counts, sizeof(h), cudaMemcpyDeviceToHost, st));
        KG_WAVE_TRY(cudaMemcpyAsync(&hq, q, sizeof(hq), cudaMemcpyDeviceToHost, st));
        KG_WAVE_TRY(cudaStreamSynchronize(st));
        for (int i = 0; i < 3; i++) {
            float ms = 0.f;
            KG_WAVE_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
            phase[i] += ms;
            total += ms;
        }
        cur ^= 1;
        if (h[cur] == 0 && h[2] == 0 && hq >= (unsigned long long)total_pairs) break;
    }
    RunCounters rc;
    KG_WAVE_TRY(cudaMemcpyAsync(&rc, ws.counters.p, sizeof(rc), cudaMemcpyDeviceToHost, st));
    KG_WAVE_TRY(cudaStreamSynchronize(st));
    stats.gh_passes = rc.gh_passes;
    stats.obj_passes = rc.obj_passes;
    stats.fp64_passes = rc.fp64_passes;
    stats.fp64_pairs = rc.fp64_pairs;
    stats.pair_sites = rc.pair_sites;
    stats.work_units = rc.work_units;
    stats.launches = launches;
    stats.flops_fp32 = rc.flops_fp32;
    stats.flops_fp64 = rc.flops_fp64;
    for (int k = 0; k < 5; k++) stats.shape_sites[k] = rc.shape_sites[k];
    stats.waves = waves;
    stats.slots = (uint64_t)n_slots;
    stats.admit_ms = phase[0];
    stats.pass_ms = phase[1];
    stats.solve_ms = phase[2];
    stats.pair_kernel_ms = total;
    if (rc.nosite_pairs) {
        err = "a pair has no jointly observed segregating site (its row is NaN)";
        return KG_ENOSITES;
    }
    return KG_OK;
}

}  // namespace kg
