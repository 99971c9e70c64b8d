// kg_engine.h — host-side engine of libkestrel_gpu.so (internal C++ API).
//
// Device-resident cohorts (bit-plane genotypes, allele frequencies of the kept
// sites) and the launch of the persistent pair kernel.  The C ABI in kg_api.cu
// is a thin layer over this.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "kestrel_gpu.h"

namespace kg {

// Owning device buffer.
// Page-locked host memory (cudaHostAlloc), grown and reused.
struct PinBuf {
    void* p = nullptr;
    size_t bytes = 0;
    PinBuf() = default;
    PinBuf(const PinBuf&) = delete;
    PinBuf& operator=(const PinBuf&) = delete;
    PinBuf(PinBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    PinBuf& operator=(PinBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~PinBuf() { release(); }
    void release();
    int reserve(size_t n);   // returns a cudaError_t
    template <class T> T* as() const { return static_cast<T*>(p); }
};

struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void release();
    // Grows to at least n bytes (contents not kept).  Returns a cudaError_t.
    int reserve(size_t n);
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// A cohort prepared on the device: allele counts, frequencies, the kept
// (segregating) sites compacted and every sample packed into {lo, hi} bit
// planes of 32 kept sites (code = 2*hi + lo; 3 = missing or padding).
struct Cohort {
    int64_t n_samples = 0;
    int64_t n_sites = 0;       // raw sites
    int64_t plane_stride = 0;  // uint2 words per sample row
    int64_t n_seg_max = 0;     // segments for n_sites (upper bound of the kept count)
    int64_t n_kept = -1;       // read back after preparation (-1 = not yet)
    DevBuf raw;                // uint8 codes, n_samples x n_sites
    DevBuf packed2, packedm;   // the last packed upload (2-bit codes, observed mask)
    DevBuf af;                 // caller frequencies, n_sites x 2 (optional)
    DevBuf rc, oc, hc;         // int32 REF allele count, observed samples, heterozygous calls
    DevBuf keep;               // uint8
    DevBuf kidx;               // int32 exclusive prefix of keep
    DevBuf bsum;               // int32 block sums of the scan
    DevBuf nkept;              // int32[2]: kept count, bad-code flag
    DevBuf pfull, qfull;       // double per raw site
    DevBuf p32;                // float REF frequency per kept site, padded to n_seg_max * 2048
    DevBuf p64, q64;           // double, same length
    DevBuf site_of;            // int32 kept index -> raw site
    DevBuf planes;             // uint2 [n_samples][plane_stride]
    bool cls = false;          // prepared for the CLS estimator (complete sites, counts over all samples)
    DevBuf cls_q;              // CLS: the 9 x 9 quadratic matrix Q, row-major double
    DevBuf cls_part;           // CLS: per-block partial sums of Q's upper triangle
    // CLS: tri- and tetra-allelic sites (the reference's gt3 / gt4)
    int64_t n_multi = 0;       // loaded sites
    int64_t n_multi_kept = -1; // sites every sample calls (read back after preparation)
    DevBuf mg;                 // uint8 genotype indices (VCF order, 255 = missing), n_samples x n_multi
    DevBuf mgT;                // the same, site-major (n_multi x n_samples)
    DevBuf malleles;           // uint8 allele count per site (3 or 4)
    DevBuf maf;                // caller frequencies, n_multi x 4 (optional)
    DevBuf mfreq;              // double frequencies used, n_multi x 4
    DevBuf mkeep;              // uint8 site used
    DevBuf mcount;             // int32[2]: sites used, bad-index flag
    DevBuf mpart;              // per-block partial sums of their Q terms
    DevBuf cmulti;             // per output row, the 9 summed rows of the pair's multi-allelic sites
    // ML: the same tri- and tetra-allelic sites after the frequency fit, the
    // maf cut and the drop of zero-frequency alleles (kg_multi.cu)
    int64_t ml_nk = 0;         // kept sites (two or more alleles remain)
    int64_t ml_stride = 0;     // bytes per sample row of ml_gr (a multiple of 32)
    int64_t ml_by_alleles[3] = {0, 0, 0};   // kept sites left with 2, 3, 4 alleles
    DevBuf ml_keep, ml_nrows, ml_kidx, ml_rbase, ml_remap, ml_redf, ml_count;   // per loaded site
    DevBuf ml_site;            // int2 per kept site: first row of its table, reduced genotypes G'
    DevBuf ml_orig;            // int32 per kept site: loaded site index
    DevBuf ml_kremap;          // uint8 [kept][10]: original genotype -> reduced genotype or ML_ZERO_ROW
    DevBuf ml_rows;            // double [rows][9]: m[g'x][g'y] of every kept site
    DevBuf ml_rows32;          // float [rows][12]: the same rows in FP32, zero-padded to three float4
    DevBuf ml_gr;              // uint8 [n_samples][ml_stride]: reduced genotype, ML_ZERO_ROW or ML_MISSING
    DevBuf ml_obs;             // uint32 [n_samples][ml_stride / 32]: called at the kept site
    size_t device_bytes() const;
};

// Enqueues the preparation of a cohort on `st`.  codes are host memory unless
// codes_on_device; af may be NULL.  maf < 0 selects 1/(2 n_samples);
// iterations caps the allele-frequency fit (the estimator's own cap).  With cls
// the sites are those every sample calls, frequencies are counts over all
// samples (or af), nothing is filtered by frequency, and Q is computed.
int prepare_cohort(Cohort& c, const uint8_t* codes, int64_t n_samples, int64_t n_sites,
                   int64_t row_stride, bool codes_on_device, const double* af, double maf,
                   cudaStream_t st, std::string& err, bool cls = false, uint64_t iterations = 100);

// After prepare_cohort(..., cls = true): adds the cohort's tri- and
// tetra-allelic sites (c.mg, c.malleles, c.maf uploaded, c.n_multi set) to the
// CLS estimator of the first num_samples samples: their frequencies (counts
// over all samples unless c.maf), Q over all sites, and each output row's
// summed rows (c.cmulti).  Sets c.n_multi_kept.
int prepare_multi(Cohort& c, bool have_af, int64_t num_samples, cudaStream_t st, std::string& err);

// Before an ML estimate: the cohort's tri- and tetra-allelic sites (c.mg,
// c.malleles, c.maf uploaded, c.n_multi set) as the reference's GL/PL path
// takes them on one-hot likelihoods (kg_multi.cu): frequencies fitted over the
// called samples (capped at `iterations`; the caller's when have_af), maf cut
// (maf < 0: 1 / (2 n_samples)), zero-frequency alleles dropped, sites with
// fewer than two alleles left discarded.  Sets c.ml_nk.
int prepare_ml_multi(Cohort& c, bool have_af, double maf, uint64_t iterations, cudaStream_t st, std::string& err);

// The GL/PL estimator on soft likelihoods of biallelic sites (kg_soft.cu): gl
// is double [n_samples][n_sites][3] on the device (linear scale, NaN =
// missing); rows of the first ns samples into d_out (device), the reference's
// order.  maf < 0: 1 / (2 n_samples).
// precision: KG_PREC_FP32C (FP32 evaluations, FP64 for pairs that need it) or
// KG_PREC_FP64; counters (5, optional): grad-Hessian evaluations, those in
// FP64, pairs escalated to FP64, pair-sites evaluated, those in FP64.
// multi (optional): tri- and tetra-allelic sites' likelihoods on the device,
// [sample][site][6] and [sample][site][10]; multi_used (3, optional): those
// kept with 2, 3 and 4 alleles after the frequency cut.
// Device buffers of the soft-likelihood estimator, kept between calls (they
// only grow, so repeated calls allocate nothing).
struct SoftWork {
    DevBuf pf, qf, keep, idx, kp, kq, ctr, g32, pq32, mgk, mgidx, mrows, mused, mscratch;
};
struct SoftMultiInput {
    const double* gl3 = nullptr;
    int64_t n3 = 0;
    const double* gl4 = nullptr;
    int64_t n4 = 0;
};
int soft_relatedness(SoftWork& w, const DevBuf& gl, int64_t n_samples, int64_t n_sites, int64_t ns,
                     uint64_t iterations, double maf, kg_output* d_out, cudaStream_t st, std::string& err,
                     int64_t* n_kept = nullptr,
                     int precision = KG_PREC_FP32C, uint64_t* counters = nullptr,
                     const SoftMultiInput* multi = nullptr, int64_t* multi_used = nullptr);

// Unpacks the VCF reader's 2-bit codes + observed mask into device byte codes
// (d2, dm: the packed rows' device copies, kept for the next load).
int unpack_2bit(DevBuf& raw, DevBuf& d2, DevBuf& dm, const uint32_t* codes2, const uint32_t* observed,
                int64_t n_samples, int64_t n_sites, cudaStream_t st, std::string& err);

// Packs query rows against a prepared panel (same raw site order); sites with
// mask[s] == 0 become missing.  Host inputs.
struct QueryPlanes {
    int64_t n_rows = 0;
    DevBuf raw;
    DevBuf mask;
    DevBuf planes;
};
int prepare_query(const Cohort& panel, QueryPlanes& q, const uint8_t* codes, int64_t n_rows,
                  int64_t row_stride, const uint8_t* site_mask, cudaStream_t st, std::string& err);

// One unit of pair work for the persistent kernel.
struct PairJob {
    const Cohort* panel = nullptr;      // frequencies, kept sites and (triangle) planes
    const QueryPlanes* query = nullptr; // rect jobs: x rows
    int kind = 0;                       // 0 triangle over panel rows, 1 rect query x panel
    int64_t n_x = 0;                    // triangle: num_samples; rect: query rows
    int64_t n_y = 0;                    // rect: panel rows
    kg_output* d_out = nullptr;         // device rows
    uint64_t iterations = 0;            // SQP iteration limit (0 = the run's); CLS: QP iterations
    int method = 0;                     // ESTIMATOR_ML or ESTIMATOR_CLS (panel prepared with cls)
    int64_t n_pairs() const { return kind == 0 ? n_x * (n_x + 1) / 2 : n_x * n_y; }
};

struct RunConfig {
    int precision = KG_PREC_FP32C;
    uint64_t iterations = 100;
    int64_t slots = 0;         // pairs in flight per wave (0 = pairs / slot_divisor within 4096..131072, as memory allows)
    int pass_blocks_per_sm = 0;   // site-pass kernel blocks per SM (0 = occupancy limit)
    uint64_t max_waves = 0;       // waves a call may run before it gives up (0 = a bound from the work)
    int ml_units = 0;             // work units per slot of the ML path's tri-/tetra-allelic sites (run_pairs sets it)
    int ml_chunk = 0;             // their kept sites per unit (run_pairs sets it)
    int unit_elems = 0;           // list entries per site-pass work unit (0 = UNIT_ELEMS, 32768)
    int slot_divisor = 5;         // automatic slots: the job's pairs / slot_divisor within 4096..131072
    // Called between waves, on the calling thread, once per job whose pairs
    // have all finished (their rows are final in device memory).
    std::function<void(int job)> job_done;
};

// Reusable device workspace of the pair engine (per-slot lists and partial
// sums, slot states, pass lists, queue, counters, cohort table).
class WaveEngine;

struct Workspace {
    DevBuf scratch, queue, counters, table;
    DevBuf partial, slots, lists_a, lists_b, tasks, counts, done;
    DevBuf ml_partial;   // per slot and unit, the sums of the ML path's tri-/tetra-allelic sites
    DevBuf qp;           // per slot the QP's inputs and solution, and the wave's list of QP slots
    PinBuf host;   // per-wave counters read back by the host loop
    int sm_count = 0;
    // run_pairs' engine, kept between calls: a call of the same shape only
    // resets its state and reuses its instantiated graphs (declared last, so
    // it goes before the buffers its graphs point into)
    std::shared_ptr<WaveEngine> engine;
};

int run_pairs(const std::vector<PairJob>& jobs, const RunConfig& cfg, Workspace& ws,
              cudaStream_t st, kg_run_stats& stats, std::string& err);

struct CohortDev;

// The wave engine (kg_wave.cu): up to n_slots pairs in flight over a job
// table that can grow between waves (the serving loop appends requests while
// others run).  open() sizes it for lists of up to list_cap entries and at most
// max_jobs jobs; add() appends jobs (their pair_begin is assigned); wave() runs
// one admit / pass / solve wave and appends the jobs whose pairs are all done
// to `finished`; idle() is true when nothing is in flight and every pair has
// been taken.
class WaveEngine {
  public:
    WaveEngine();
    ~WaveEngine();
    WaveEngine(const WaveEngine&) = delete;
    WaveEngine& operator=(const WaveEngine&) = delete;
    int open(Workspace& ws, cudaStream_t st, const RunConfig& cfg, int64_t list_cap, int64_t expected_pairs,
             int max_jobs, std::string& err);
    int add(const std::vector<CohortDev>& jobs, std::string& err);
    int wave(std::vector<int>& finished, std::string& err);
    // Runs waves until the engine is idle inside one graph launch (a device
    // loop: no host round trip per wave), at most max_waves of them.
    int run_until_idle(unsigned long long max_waves, std::string& err);
    bool idle() const;
    int64_t n_slots() const;
    int64_t list_cap() const;
    // Pairs of the table that no slot has taken yet.
    int64_t backlog() const;
    // Empties the job table (only when idle), so a long-running loop reuses it.
    int reset_jobs(std::string& err);
    // Counters and phase times since open().
    int stats(kg_run_stats& stats, std::string& err);

  private:
    struct Impl;
    Impl* d_;
};

// The device table entry of a job (pair_begin left 0 for the engine to set),
// and the list capacity (entries per slot) a cohort's pairs need.
CohortDev make_cohort_dev(const PairJob& jb, uint64_t iterations);
int64_t list_capacity(const Cohort& panel);

// All jobs of one call through one engine (kg_wave.cu), over a prepared
// cohort table.
int run_waves(const std::vector<PairJob>& jobs, const RunConfig& cfg, Workspace& ws, cudaStream_t st,
              kg_run_stats& stats, std::string& err, const std::vector<CohortDev>& table,
              int64_t total_pairs, int64_t list_cap);


const char* engine_version();

// Measured FFMA throughput (TFLOP/s).
int fp32_peak(int device, double& tflops, std::string& err);

}  // namespace kg
