// kg_api.cu — extern "C" boundary of libkestrel_gpu.so (see include/kestrel_gpu.h).
//
// No exception or CUDA error crosses this boundary: every entry point returns a
// kg_status and records a message for kg_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "kestrel_gpu.h"
#include "kg_engine.h"
#include "kg_pair.cuh"

namespace {

struct Request {
    int64_t id = 0;
    int64_t n_query = 0;
    uint64_t iterations = 100;
    std::vector<uint8_t> codes;   // n_query x n_sites
    std::vector<uint8_t> mask;    // n_sites or empty
    std::vector<kg_output> rows;
    int status = KG_OK;
    std::string err;
    bool done = false;
    bool cancelled = false;
};

}  // namespace

struct kg_ctx {
    int device = 0;
    size_t budget = 0;
    int precision = KG_PREC_FP32C;
    int64_t wave_slots = 0;
    int pass_bps = 0;
    int unit_elems = 0;
    int slot_divisor = 5;
    uint64_t wave_limit = 0;
    cudaStream_t stream = nullptr;
    // single cohort
    kg::Cohort cohort;
    bool loaded = false;
    std::vector<double> af;
    bool af_set = false;
    bool multi_af = false;                // kg_load_multiallelic gave frequencies
    kg::DevBuf soft_gl;                   // kg_load_likelihoods: double [sample][site][3]
    int64_t soft_ns = 0, soft_nv = 0;
    kg::DevBuf soft_gl3, soft_gl4;        // kg_load_likelihoods_multiallelic: [sample][site][6], [..][10]
    kg::SoftWork soft_work;               // the soft estimator's buffers, kept between calls
    int64_t soft_n3 = 0, soft_n4 = 0;
    kg::Workspace ws;
    kg::DevBuf dout;
    kg_run_stats last{};
    // serving
    std::mutex mu;
    std::condition_variable cv;
    std::vector<std::thread> servers;
    bool stop = false;
    bool panel_ready = false;
    kg::Cohort panel;
    std::map<int64_t, std::shared_ptr<Request>> requests;
    std::deque<int64_t> pending;
    int64_t next_id = 1;
    int64_t served_requests = 0, served_pairs = 0, served_launches = 0;
    int64_t in_flight = 0;               // requests admitted into a serving engine
    int64_t panel_gen = 0;               // bumped by every kg_panel_load
    struct ServeWorker {
        cudaStream_t stream = nullptr;
        kg::Workspace ws;
    };
    std::vector<ServeWorker> workers;
};

namespace {

// The message of the calling thread's last failing call: serving calls run on
// several threads at once, so each thread keeps its own.
thread_local std::string t_last_err;

int set_err(kg_ctx* c, int st, const std::string& msg) {
    (void)c;
    t_last_err = msg;
    return st;
}

int use_device(kg_ctx* c) {
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return KG_OK;
}

bool budget_ok(kg_ctx* c, size_t extra) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return false;
    if (extra > fr) return false;
    if (c->budget) {
        size_t used = tot - fr;
        if (used + extra > c->budget) return false;
    }
    return true;
}

template <class F>
int guarded(kg_ctx* c, F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        return set_err(c, KG_ENOMEM, "host allocation failed");
    } catch (const std::exception& ex) {
        return set_err(c, KG_ECUDA, ex.what());
    } catch (...) {
        return set_err(c, KG_ECUDA, "unknown error");
    }
}

kg::RunConfig run_config(const kg_ctx* c, uint64_t iterations) {
    kg::RunConfig cfg;
    cfg.precision = c->precision;
    cfg.iterations = iterations;
    cfg.slots = c->wave_slots;
    cfg.pass_blocks_per_sm = c->pass_bps;
    cfg.max_waves = c->wave_limit;
    cfg.unit_elems = c->unit_elems;
    cfg.slot_divisor = c->slot_divisor;
    return cfg;
}

int copy_rows_out(kg_ctx* c, const kg::DevBuf& d, int64_t n, kg_output* out, cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(out, d.p, sizeof(kg_output) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("copy rows: ") + cudaGetErrorString(e));
    return KG_OK;
}

// ------------------------------------------------------------- serving loop

// Requests in the engine's job table between idle moments; when it fills, new
// requests wait until the in-flight ones drain.
constexpr int kMaxServeJobs = 1 << 16;

// One request in the serving engine: its query planes and device rows live
// until its last pair is done.
struct LiveRequest {
    std::shared_ptr<Request> r;
    std::unique_ptr<kg::QueryPlanes> q;
    kg_output* d_out = nullptr;
};

// Serving workers, each with its own stream and wave engine; their kernels
// overlap on the device.
constexpr int kServeWorkers = 2;
// Pairs in flight per worker (as memory allows).
constexpr int64_t kServeSlots = 32768;
// A worker takes more requests only while fewer than this many of its pairs
// wait for a slot (its slots stay busy; a burst spreads over the workers).
constexpr int64_t kWorkerBacklog = 1 << 16;

// One serving worker.  Its wave engine runs while it has requests in flight.
// Between waves, queued requests whose inputs and rows fit the memory budget
// join the engine's job table, so their pairs take slots as slots free
// (continuous batching); a request is answered as soon as its own pairs are
// done.  A pair's result does not depend on which requests share its waves.
void serve_loop(kg_ctx* c, int wid) {
    cudaSetDevice(c->device);
    const cudaStream_t st = c->workers[wid].stream;
    kg::Workspace& wws = c->workers[wid].ws;
    int64_t my_backlog = 0;   // pairs of this worker's requests not yet in a slot
    std::unique_ptr<kg::WaveEngine> eng;   // (re)opened for each panel
    int64_t eng_gen = -1;
    std::map<int, LiveRequest> live;     // by job index
    int next_job = 0;
    std::string err;
    auto fail_all = [&](int status, const std::string& why) {
        std::lock_guard<std::mutex> lk(c->mu);
        for (auto& kv : live) {
            kv.second.r->status = status;
            kv.second.r->err = why;
            kv.second.r->done = true;
            if (kv.second.d_out) cudaFreeAsync(kv.second.d_out, st);
        }
        c->in_flight -= (int64_t)live.size();
        live.clear();
        my_backlog = 0;
        c->cv.notify_all();
    };
    for (;;) {
        std::vector<std::shared_ptr<Request>> admit;
        {
            std::unique_lock<std::mutex> lk(c->mu);
            c->cv.wait(lk, [&] { return c->stop || !live.empty() || !c->pending.empty(); });
            if (c->stop) {
                for (int64_t id : c->pending) {
                    auto it = c->requests.find(id);
                    if (it != c->requests.end()) {
                        it->second->status = KG_ECANCELED;
                        it->second->done = true;
                    }
                }
                c->pending.clear();
                c->cv.notify_all();
                lk.unlock();
                fail_all(KG_ECANCELED, "context destroyed");
                break;
            }
            // the queued requests that fit, in arrival order
            size_t bytes = 0;
            int64_t take = my_backlog;
            while (!c->pending.empty() && next_job + (int)admit.size() < kMaxServeJobs &&
                   (admit.empty() && live.empty() ? true : take < kWorkerBacklog)) {
                const int64_t id = c->pending.front();
                auto it = c->requests.find(id);
                if (it == c->requests.end() || it->second->cancelled) {
                    c->pending.pop_front();
                    continue;
                }
                auto& r = it->second;
                const size_t nb = (size_t)(r->n_query * c->panel.n_samples) * sizeof(kg_output) +
                                  (size_t)r->n_query * (size_t)(c->panel.n_sites + c->panel.plane_stride * 8);
                if ((!admit.empty() || !live.empty()) && !budget_ok(c, bytes + nb)) break;
                admit.push_back(r);
                bytes += nb;
                take += r->n_query * c->panel.n_samples;
                c->pending.pop_front();
            }
            c->in_flight += (int64_t)admit.size();
        }
        if (!eng || (eng_gen != c->panel_gen && live.empty())) {
            // a new panel (kg_panel_load waits for in-flight requests first)
            eng = std::make_unique<kg::WaveEngine>();
            next_job = 0;
            kg::RunConfig cfg = run_config(c, 100);
            if (cfg.slots == 0) cfg.slots = kServeSlots;
            const int r = eng->open(wws, st, cfg, kg::list_capacity(c->panel), (int64_t)1 << 40,
                                    kMaxServeJobs, err);
            if (r) {
                eng.reset();
                std::lock_guard<std::mutex> lk(c->mu);
                for (auto& rq : admit) { rq->status = r; rq->err = err; rq->done = true; }
                c->in_flight -= (int64_t)admit.size();
                c->cv.notify_all();
                continue;
            }
            eng_gen = c->panel_gen;
        }
        // the admitted requests join the engine
        std::vector<kg::CohortDev> add;
        for (auto& rq : admit) {
            LiveRequest lr;
            lr.r = rq;
            lr.q = std::make_unique<kg::QueryPlanes>();
            const int64_t np = rq->n_query * c->panel.n_samples;
            int r = kg::prepare_query(c->panel, *lr.q, rq->codes.data(), rq->n_query, c->panel.n_sites,
                                      rq->mask.empty() ? nullptr : rq->mask.data(), st, err);
            if (r == KG_OK && cudaMallocAsync(reinterpret_cast<void**>(&lr.d_out), sizeof(kg_output) * np, st) !=
                                  cudaSuccess) {
                r = KG_ENOMEM;
                err = "request rows do not fit";
                lr.d_out = nullptr;
            }
            if (r != KG_OK) {
                std::lock_guard<std::mutex> lk(c->mu);
                rq->status = r;
                rq->err = err;
                rq->done = true;
                c->in_flight--;
                c->cv.notify_all();
                continue;
            }
            kg::PairJob jb;
            jb.panel = &c->panel;
            jb.query = lr.q.get();
            jb.kind = 1;
            jb.n_x = rq->n_query;
            jb.n_y = c->panel.n_samples;
            jb.d_out = lr.d_out;
            jb.iterations = rq->iterations;   // each request keeps its own limit
            add.push_back(kg::make_cohort_dev(jb, rq->iterations));
            live[next_job++] = std::move(lr);
        }
        int r = add.empty() ? KG_OK : eng->add(add, err);
        std::vector<int> fin;
        if (r == KG_OK && !eng->idle()) {
            r = eng->wave(fin, err);
            std::lock_guard<std::mutex> lk(c->mu);
            c->served_launches++;
        }
        if (r != KG_OK) {
            // the engine's state is unknown after a failure: start a new one
            fail_all(r, err);
            eng.reset();
            continue;
        }
        // answer the requests whose pairs are all done
        for (int j : fin) {
            auto it = live.find(j);
            if (it == live.end()) continue;
            LiveRequest& lr = it->second;
            const int64_t np = lr.r->n_query * c->panel.n_samples;
            lr.r->rows.resize(np);
            cudaError_t ce = cudaMemcpyAsync(lr.r->rows.data(), lr.d_out, sizeof(kg_output) * np,
                                             cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaFreeAsync(lr.d_out, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            std::lock_guard<std::mutex> lk(c->mu);
            if (ce != cudaSuccess) {
                lr.r->status = KG_ECUDA;
                lr.r->err = cudaGetErrorString(ce);
            }
            lr.r->done = true;
            c->served_requests++;
            c->served_pairs += np;
            c->in_flight--;
            c->cv.notify_all();
            live.erase(it);
        }
        my_backlog = eng ? eng->backlog() : 0;
        if (eng->idle() && live.empty() && next_job > 0) {
            std::string e2;
            if (eng->reset_jobs(e2) == KG_OK) next_job = 0;
            else eng.reset();
        }
    }
}

}  // namespace

extern "C" {

const char* kg_version(void) { return kg::engine_version(); }

int kg_create(kg_ctx** ctx, int device, size_t mem_budget) {
    if (!ctx) return KG_EINVAL;
    *ctx = nullptr;
    kg_ctx* c = new (std::nothrow) kg_ctx();
    if (!c) return KG_ENOMEM;
    c->device = device;
    c->budget = mem_budget;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        delete c;
        return KG_ECUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return KG_ECUDA;
    }
    *ctx = c;
    return KG_OK;
}

int kg_destroy(kg_ctx* c) {
    if (!c) return KG_EINVAL;
    cudaSetDevice(c->device);
    {
        std::lock_guard<std::mutex> lk(c->mu);
        c->stop = true;
        c->cv.notify_all();
    }
    for (auto& t : c->servers)
        if (t.joinable()) t.join();
    for (auto& w : c->workers)
        if (w.stream) {
            cudaStreamSynchronize(w.stream);
            cudaStreamDestroy(w.stream);
        }
    if (c->stream) {
        cudaStreamSynchronize(c->stream);
        cudaStreamDestroy(c->stream);
    }
    delete c;
    return KG_OK;
}

const char* kg_last_error(const kg_ctx* c) { return c ? t_last_err.c_str() : "null context"; }

int kg_set_precision(kg_ctx* c, int precision) {
    if (!c || (precision != KG_PREC_FP32C && precision != KG_PREC_FP64)) return set_err(c, KG_EINVAL, "precision must be KG_PREC_FP32C or KG_PREC_FP64");
    c->precision = precision;
    return KG_OK;
}

int kg_set_launch(kg_ctx* c, int slots, int blocks_per_sm) {
    if (!c || slots < 0 || slots > (1 << 20) || blocks_per_sm < 0 || blocks_per_sm > 32)
        return set_err(c, KG_EINVAL, "slots must be 0..2^20 and blocks_per_sm 0..32");
    c->wave_slots = slots;
    c->pass_bps = blocks_per_sm;
    return KG_OK;
}

int kg_set_work_unit(kg_ctx* c, int entries) {
    if (!c) return KG_EINVAL;
    if (entries != 0 && (entries < 1024 || entries > 65536 || entries % 512 != 0))
        return set_err(c, KG_EINVAL, "the work unit must be 0 or a multiple of 512 from 1024 to 65536 entries");
    c->unit_elems = entries;
    return KG_OK;
}

int kg_get_launch(const kg_ctx* c, int* slots, int* blocks_per_sm, int* unit_entries, int* slot_divisor) {
    if (!c) return KG_EINVAL;
    if (slots) *slots = (int)c->wave_slots;
    if (blocks_per_sm) *blocks_per_sm = c->pass_bps;
    if (unit_entries) *unit_entries = c->unit_elems;
    if (slot_divisor) *slot_divisor = c->slot_divisor;
    return KG_OK;
}

int kg_set_wave_limit(kg_ctx* c, uint64_t waves) {
    if (!c) return KG_EINVAL;
    c->wave_limit = waves;
    return KG_OK;
}

int kg_load_genotypes(kg_ctx* c, const uint8_t* codes, int64_t n_samples, int64_t n_sites,
                      int64_t row_stride) {
    if (!c) return KG_EINVAL;
    if (!codes || n_samples <= 0 || n_sites <= 0 || row_stride < n_sites)
        return set_err(c, KG_EINVAL, "codes must be non-NULL with n_samples, n_sites > 0 and row_stride >= n_sites");
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        if (!budget_ok(c, (size_t)(n_samples * n_sites))) return set_err(c, KG_ENOMEM, "genotypes exceed the memory budget");
        if (c->cohort.raw.reserve((size_t)(n_samples * n_sites)) != cudaSuccess)
            return set_err(c, KG_ENOMEM, "cannot allocate device genotypes");
        cudaError_t e = cudaMemcpy2DAsync(c->cohort.raw.p, (size_t)n_sites, codes, (size_t)row_stride,
                                          (size_t)n_sites, (size_t)n_samples, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("upload: ") + cudaGetErrorString(e));
        c->cohort.n_samples = n_samples;
        c->cohort.n_sites = n_sites;
        c->cohort.n_kept = -1;
        c->cohort.n_multi = 0;
        c->loaded = true;
        c->af_set = false;
        return KG_OK;
    });
}

int kg_load_genotypes_2bit(kg_ctx* c, const uint32_t* codes2, const uint32_t* observed,
                           int64_t n_samples, int64_t n_sites) {
    if (!c) return KG_EINVAL;
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        std::string err;
        st = kg::unpack_2bit(c->cohort.raw, c->cohort.packed2, c->cohort.packedm, codes2, observed, n_samples,
                             n_sites, c->stream, err);
        if (st) return set_err(c, st, err);
        c->cohort.n_samples = n_samples;
        c->cohort.n_sites = n_sites;
        c->cohort.n_kept = -1;
        c->cohort.n_multi = 0;
        c->loaded = true;
        c->af_set = false;
        return KG_OK;
    });
}

int kg_load_multiallelic(kg_ctx* c, const uint8_t* gidx, int64_t n_samples, int64_t n_sites, int64_t row_stride,
                         const uint8_t* n_alleles, const double* af) {
    if (!c) return KG_EINVAL;
    if (!c->loaded) return set_err(c, KG_EINVAL, "load genotypes first");
    if (n_sites == 0) {
        c->cohort.n_multi = 0;
        return KG_OK;
    }
    if (!gidx || !n_alleles || n_sites < 0 || row_stride < n_sites)
        return set_err(c, KG_EINVAL, "gidx and n_alleles must be non-NULL with n_sites > 0 and row_stride >= n_sites");
    if (n_samples != c->cohort.n_samples)
        return set_err(c, KG_EINVAL, "n_samples must match the loaded genotypes");
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        kg::Cohort& co = c->cohort;
        if (!budget_ok(c, (size_t)(n_samples * n_sites)))
            return set_err(c, KG_ENOMEM, "multi-allelic genotypes exceed the memory budget");
        if (co.mg.reserve((size_t)(n_samples * n_sites)) != cudaSuccess || co.malleles.reserve((size_t)n_sites) != cudaSuccess ||
            (af && co.maf.reserve(sizeof(double) * 4 * n_sites) != cudaSuccess))
            return set_err(c, KG_ENOMEM, "cannot allocate device multi-allelic genotypes");
        cudaError_t e = cudaMemcpy2DAsync(co.mg.p, (size_t)n_sites, gidx, (size_t)row_stride, (size_t)n_sites,
                                          (size_t)n_samples, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(co.malleles.p, n_alleles, (size_t)n_sites, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess && af)
            e = cudaMemcpyAsync(co.maf.p, af, sizeof(double) * 4 * n_sites, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("upload: ") + cudaGetErrorString(e));
        co.n_multi = n_sites;
        c->multi_af = af != nullptr;
        return KG_OK;
    });
}

int kg_set_allele_frequencies(kg_ctx* c, const double* af) {
    if (!c) return KG_EINVAL;
    if (!c->loaded) return set_err(c, KG_EINVAL, "load genotypes first");
    return guarded(c, [&]() -> int {
        if (!af) {
            c->af.clear();
            c->af_set = false;
            return KG_OK;
        }
        c->af.assign(af, af + 2 * c->cohort.n_sites);
        c->af_set = true;
        return KG_OK;
    });
}

int kg_relatedness(kg_ctx* c, int64_t num_samples, uint64_t iterations, double maf, kg_output* out,
                   int64_t out_cap, int64_t* n_out) {
    if (!c) return KG_EINVAL;
    if (!c->loaded) return set_err(c, KG_EINVAL, "no genotypes loaded");
    if (iterations == 0) return set_err(c, KG_EINVAL, "iterations must be non-zero");
    if (!(std::isnan(maf) || maf < 0.0) && maf > 1.0)
        return set_err(c, KG_EINVAL, "Minimum allele frequency must be within 0 to 1");
    int64_t ns = num_samples < 0 ? c->cohort.n_samples : num_samples;
    if (ns == 0) return set_err(c, KG_EINVAL, "num_samples must be positive (or negative for all samples)");
    if (ns > c->cohort.n_samples)
        return set_err(c, KG_EINVAL, "Requested samples " + std::to_string(ns) + " exceeds total samples " +
                                         std::to_string(c->cohort.n_samples));
    int64_t np = ns * (ns + 1) / 2;
    if (!out || out_cap < np) return set_err(c, KG_EINVAL, "output capacity must be at least num_samples*(num_samples+1)/2");
    return guarded(c, [&]() -> int {
        auto t0 = std::chrono::steady_clock::now();
        int st = use_device(c);
        if (st) return st;
        std::string err;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, c->stream);
        st = kg::prepare_cohort(c->cohort, c->cohort.raw.as<uint8_t>(), c->cohort.n_samples,
                                c->cohort.n_sites, c->cohort.n_sites, true,
                                c->af_set ? c->af.data() : nullptr, std::isnan(maf) ? -1.0 : maf,
                                c->stream, err, false, iterations);
        if (!st)
            st = kg::prepare_ml_multi(c->cohort, c->multi_af, std::isnan(maf) ? -1.0 : maf, iterations, c->stream,
                                      err);
        if (st) {
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
            return set_err(c, st, err);
        }
        if (c->dout.reserve(sizeof(kg_output) * np) != cudaSuccess)
            return set_err(c, KG_ENOMEM, "cannot allocate device output rows");
        kg::PairJob jb;
        jb.panel = &c->cohort;
        jb.kind = 0;
        jb.n_x = ns;
        jb.d_out = c->dout.as<kg_output>();
        std::vector<kg::PairJob> jobs{jb};
        kg_run_stats stats{};
        st = kg::run_pairs(jobs, run_config(c, iterations), c->ws, c->stream, stats, err);
        cudaEventRecord(ev1, c->stream);
        int st2 = copy_rows_out(c, c->dout, np, out, c->stream);
        float dms = 0.f;
        if (cudaEventElapsedTime(&dms, ev0, ev1) == cudaSuccess) stats.device_ms = dms;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        stats.launches += 7;  // count, freq, two scans, compact, pad, pack
        const kg::Cohort& co = c->cohort;
        if (co.n_multi > 0) stats.launches += 3 + (co.ml_nk > 0 ? 2 : 0);   // fit, two scans, rows, codes
        stats.sites_used[0] = (uint64_t)(co.n_kept + co.ml_by_alleles[0]);
        stats.sites_used[1] = (uint64_t)co.ml_by_alleles[1];
        stats.sites_used[2] = (uint64_t)co.ml_by_alleles[2];
        stats.sites_discarded = (uint64_t)(co.n_sites + co.n_multi - co.n_kept - co.ml_nk);
        if (st2 && !st) st = st2;
        stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        c->last = stats;
        if (n_out) *n_out = np;
        if (st) return set_err(c, st, err.empty() ? t_last_err : err);
        return KG_OK;
    });
}

// The reference's default hard-call estimator, conditional least squares with
// the Brier objective (calculate_relatedness_coefficients_gt,
// src/wrapper.rs:22-29 -> src/coefficients.rs:166-278): the cohort is prepared
// with the GT reader's site rule and count frequencies, then every pair takes
// one CLS moment pass and the simplex QP in the wave engine.
int kg_relatedness_gt(kg_ctx* c, int64_t num_samples, uint64_t iterations, kg_output* out, int64_t out_cap,
                      int64_t* n_out) {
    if (!c) return KG_EINVAL;
    if (!c->loaded) return set_err(c, KG_EINVAL, "no genotypes loaded");
    if (iterations == 0) return set_err(c, KG_EINVAL, "iterations must be non-zero");
    int64_t ns = num_samples < 0 ? c->cohort.n_samples : num_samples;
    if (ns == 0) return set_err(c, KG_EINVAL, "num_samples must be positive (or negative for all samples)");
    if (ns > c->cohort.n_samples)
        return set_err(c, KG_EINVAL, "Requested samples " + std::to_string(ns) + " exceeds total samples " +
                                         std::to_string(c->cohort.n_samples));
    int64_t np = ns * (ns + 1) / 2;
    if (!out || out_cap < np) return set_err(c, KG_EINVAL, "output capacity must be at least num_samples*(num_samples+1)/2");
    return guarded(c, [&]() -> int {
        auto t0 = std::chrono::steady_clock::now();
        int st = use_device(c);
        if (st) return st;
        std::string err;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, c->stream);
        st = kg::prepare_cohort(c->cohort, c->cohort.raw.as<uint8_t>(), c->cohort.n_samples,
                                c->cohort.n_sites, c->cohort.n_sites, true,
                                c->af_set ? c->af.data() : nullptr, -1.0, c->stream, err, true);
        if (!st) st = kg::prepare_multi(c->cohort, c->multi_af, ns, c->stream, err);
        if (st) {
            cudaEventDestroy(ev0);
            cudaEventDestroy(ev1);
            return set_err(c, st, err);
        }
        if (c->dout.reserve(sizeof(kg_output) * np) != cudaSuccess)
            return set_err(c, KG_ENOMEM, "cannot allocate device output rows");
        kg::PairJob jb;
        jb.panel = &c->cohort;
        jb.kind = 0;
        jb.n_x = ns;
        jb.d_out = c->dout.as<kg_output>();
        jb.method = kg::ESTIMATOR_CLS;
        std::vector<kg::PairJob> jobs{jb};
        kg_run_stats stats{};
        st = kg::run_pairs(jobs, run_config(c, iterations), c->ws, c->stream, stats, err);
        cudaEventRecord(ev1, c->stream);
        int st2 = copy_rows_out(c, c->dout, np, out, c->stream);
        float dms = 0.f;
        if (cudaEventElapsedTime(&dms, ev0, ev1) == cudaSuccess) stats.device_ms = dms;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        stats.launches += 9;  // count, freq, two scans, compact, pad, pack, Gram, Gram total
        if (c->cohort.n_multi > 0) stats.launches += 5;   // multi-allelic frequencies, Gram, Gram total, transpose, rows
        stats.sites_used[0] = (uint64_t)c->cohort.n_kept;
        stats.sites_discarded = (uint64_t)(c->cohort.n_sites - c->cohort.n_kept +
                                           (c->cohort.n_multi > 0 ? c->cohort.n_multi - c->cohort.n_multi_kept : 0));
        if (st2 && !st) st = st2;
        stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        c->last = stats;
        if (n_out) *n_out = np;
        if (st) return set_err(c, st, err.empty() ? t_last_err : err);
        return KG_OK;
    });
}

int kg_load_likelihoods(kg_ctx* c, const double* gl, int64_t n_samples, int64_t n_sites) {
    if (!c) return KG_EINVAL;
    if (!gl || n_samples <= 0 || n_sites <= 0 || n_sites > (int64_t)INT32_MAX)
        return set_err(c, KG_EINVAL, "gl must be non-NULL with n_samples, n_sites > 0");
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        const size_t bytes = sizeof(double) * 3 * (size_t)n_samples * (size_t)n_sites;
        if (!budget_ok(c, bytes)) return set_err(c, KG_ENOMEM, "likelihoods exceed the memory budget");
        if (c->soft_gl.reserve(bytes) != cudaSuccess) return set_err(c, KG_ENOMEM, "cannot allocate device likelihoods");
        cudaError_t e = cudaMemcpyAsync(c->soft_gl.p, gl, bytes, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("upload: ") + cudaGetErrorString(e));
        c->soft_ns = n_samples;
        c->soft_nv = n_sites;
        c->soft_n3 = 0;
        c->soft_n4 = 0;
        return KG_OK;
    });
}

int kg_load_likelihoods_multiallelic(kg_ctx* c, const double* gl, int64_t n_samples, int64_t n_sites,
                                     int n_alleles) {
    if (!c) return KG_EINVAL;
    if (!c->soft_ns) return set_err(c, KG_EINVAL, "load the biallelic likelihoods first");
    if (n_alleles != 3 && n_alleles != 4) return set_err(c, KG_EINVAL, "n_alleles must be 3 or 4");
    if (n_samples != c->soft_ns) return set_err(c, KG_EINVAL, "n_samples must match the loaded likelihoods");
    if (n_sites < 0 || n_sites > (int64_t)INT32_MAX || (n_sites > 0 && !gl))
        return set_err(c, KG_EINVAL, "gl must be non-NULL with n_sites >= 0");
    int64_t& count = n_alleles == 3 ? c->soft_n3 : c->soft_n4;
    kg::DevBuf& buf = n_alleles == 3 ? c->soft_gl3 : c->soft_gl4;
    if (n_sites == 0) {
        count = 0;
        return KG_OK;
    }
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        const int ng = n_alleles * (n_alleles + 1) / 2;
        const size_t bytes = sizeof(double) * ng * (size_t)n_samples * (size_t)n_sites;
        if (!budget_ok(c, bytes)) return set_err(c, KG_ENOMEM, "likelihoods exceed the memory budget");
        if (buf.reserve(bytes) != cudaSuccess) return set_err(c, KG_ENOMEM, "cannot allocate device likelihoods");
        cudaError_t e = cudaMemcpyAsync(buf.p, gl, bytes, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("upload: ") + cudaGetErrorString(e));
        count = n_sites;
        return KG_OK;
    });
}

int kg_relatedness_gl(kg_ctx* c, int64_t num_samples, uint64_t iterations, double maf, kg_output* out,
                      int64_t out_cap, int64_t* n_out) {
    if (!c) return KG_EINVAL;
    if (!c->soft_ns) return set_err(c, KG_EINVAL, "no likelihoods loaded");
    if (iterations == 0) return set_err(c, KG_EINVAL, "iterations must be non-zero");
    if (!(std::isnan(maf) || maf < 0.0) && maf > 1.0)
        return set_err(c, KG_EINVAL, "Minimum allele frequency must be within 0 to 1");
    const int64_t ns = num_samples < 0 ? c->soft_ns : num_samples;
    if (ns == 0) return set_err(c, KG_EINVAL, "num_samples must be positive (or negative for all samples)");
    if (ns > c->soft_ns)
        return set_err(c, KG_EINVAL, "Requested samples " + std::to_string(ns) + " exceeds total samples " +
                                         std::to_string(c->soft_ns));
    const int64_t np = ns * (ns + 1) / 2;
    if (!out || out_cap < np) return set_err(c, KG_EINVAL, "output capacity must be at least num_samples*(num_samples+1)/2");
    return guarded(c, [&]() -> int {
        auto t0 = std::chrono::steady_clock::now();
        int st = use_device(c);
        if (st) return st;
        if (c->dout.reserve(sizeof(kg_output) * np) != cudaSuccess)
            return set_err(c, KG_ENOMEM, "cannot allocate device output rows");
        std::string err;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, c->stream);
        int64_t kept = 0, used[3] = {0, 0, 0};
        uint64_t sc[5] = {0, 0, 0, 0, 0};
        kg::SoftMultiInput mi;
        mi.gl3 = c->soft_n3 ? c->soft_gl3.as<double>() : nullptr;
        mi.n3 = c->soft_n3;
        mi.gl4 = c->soft_n4 ? c->soft_gl4.as<double>() : nullptr;
        mi.n4 = c->soft_n4;
        st = kg::soft_relatedness(c->soft_work, c->soft_gl, c->soft_ns, c->soft_nv, ns, iterations, std::isnan(maf) ? -1.0 : maf,
                                  c->dout.as<kg_output>(), c->stream, err, &kept, c->precision, sc, &mi, used);
        cudaEventRecord(ev1, c->stream);
        int st2 = copy_rows_out(c, c->dout, np, out, c->stream);
        kg_run_stats stats{};
        float dms = 0.f;
        if (cudaEventElapsedTime(&dms, ev0, ev1) == cudaSuccess) stats.device_ms = dms;
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        stats.launches = c->precision == KG_PREC_FP64 ? 2 : 3;   // frequencies, (FP32 packing,) pairs
        stats.gh_passes = sc[0];
        stats.obj_passes = sc[0];
        stats.fp64_passes = sc[1];
        stats.fp64_pairs = sc[2];
        stats.work_units = sc[3];
        // executed FP32 arithmetic at 204 FLOP per pair-site (FMA = 2): the
        // row from the nine likelihood products, d, the gradient and the 45
        // Hessian terms, the objective term
        stats.flops_fp32 = (sc[3] - sc[4]) * 204ull;
        stats.sites_used[0] = (uint64_t)(kept + used[0]);
        stats.sites_used[1] = (uint64_t)used[1];
        stats.sites_used[2] = (uint64_t)used[2];
        stats.sites_discarded = (uint64_t)(c->soft_nv + c->soft_n3 + c->soft_n4 - kept - used[0] - used[1] - used[2]);
        stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        c->last = stats;
        if (n_out) *n_out = np;
        if (!st && st2) st = st2;
        if (st) return set_err(c, st, err.empty() ? t_last_err : err);
        return KG_OK;
    });
}

int kg_relatedness_coefficients(const uint8_t* codes, int64_t n_samples, int64_t n_sites,
                                int64_t row_stride, const double* allele_frequencies, int64_t threads,
                                uint64_t iterations, double maf, int64_t num_samples, kg_output* out,
                                int64_t out_cap, int64_t* n_out) {
    (void)threads;
    kg_ctx* c = nullptr;
    int st = kg_create(&c, 0, 0);
    if (st) return st;
    st = kg_load_genotypes(c, codes, n_samples, n_sites, row_stride);
    if (!st && allele_frequencies) st = kg_set_allele_frequencies(c, allele_frequencies);
    if (!st) st = kg_relatedness(c, num_samples, iterations, maf, out, out_cap, n_out);
    kg_destroy(c);
    return st;
}

int kg_relatedness_batch(kg_ctx* c, kg_cohort* cohorts, int n_cohorts, uint64_t iterations, double maf) {
    if (!c) return KG_EINVAL;
    if (!cohorts || n_cohorts <= 0) return set_err(c, KG_EINVAL, "no cohorts");
    if (iterations == 0) return set_err(c, KG_EINVAL, "iterations must be non-zero");
    return guarded(c, [&]() -> int {
        auto t0 = std::chrono::steady_clock::now();
        int st = use_device(c);
        if (st) return st;
        std::vector<std::unique_ptr<kg::Cohort>> prep;
        std::vector<kg::PairJob> jobs;
        std::vector<int> job_of(n_cohorts, -1);
        std::vector<int64_t> offs(n_cohorts, 0);
        int64_t total = 0;
        std::string err;
        for (int i = 0; i < n_cohorts; i++) {
            kg_cohort& k = cohorts[i];
            k.n_out = 0;
            int64_t ns = k.num_samples < 0 ? k.n_samples : k.num_samples;
            if (!k.codes || ns <= 0 || ns > k.n_samples || !k.out || k.out_cap < ns * (ns + 1) / 2) {
                k.status = KG_EINVAL;
                continue;
            }
            auto co = std::make_unique<kg::Cohort>();
            std::string e1;
            int s1 = kg::prepare_cohort(*co, k.codes, k.n_samples, k.n_sites, k.row_stride, false,
                                        k.allele_frequencies, std::isnan(maf) ? -1.0 : maf, c->stream, e1, false,
                                        iterations);
            k.status = s1;
            if (s1) {
                if (err.empty()) err = e1;
                continue;
            }
            co->raw.release();  // packed planes are all the pair kernel needs
            kg::PairJob jb;
            jb.panel = co.get();
            jb.kind = 0;
            jb.n_x = ns;
            offs[i] = total;
            total += jb.n_pairs();
            job_of[i] = (int)jobs.size();
            jobs.push_back(jb);
            prep.push_back(std::move(co));
        }
        if (jobs.empty()) return set_err(c, KG_EINVAL, err.empty() ? "no valid cohort" : err);
        if (c->dout.reserve(sizeof(kg_output) * total) != cudaSuccess)
            return set_err(c, KG_ENOMEM, "cannot allocate device output rows");
        for (int i = 0; i < n_cohorts; i++)
            if (job_of[i] >= 0) jobs[job_of[i]].d_out = c->dout.as<kg_output>() + offs[i];
        kg_run_stats stats{};
        st = kg::run_pairs(jobs, run_config(c, iterations), c->ws, c->stream, stats, err);
        for (int i = 0; i < n_cohorts; i++) {
            if (job_of[i] < 0) continue;
            int64_t np = jobs[job_of[i]].n_pairs();
            cudaError_t e = cudaMemcpyAsync(cohorts[i].out, c->dout.as<kg_output>() + offs[i],
                                            sizeof(kg_output) * np, cudaMemcpyDeviceToHost, c->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
            if (e != cudaSuccess) return set_err(c, KG_ECUDA, std::string("copy rows: ") + cudaGetErrorString(e));
            cohorts[i].n_out = np;
            if (st == KG_ENOSITES) {
                for (int64_t r = 0; r < np; r++)
                    if (std::isnan(cohorts[i].out[r].obj)) { cohorts[i].status = KG_ENOSITES; break; }
            }
        }
        stats.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        c->last = stats;
        if (st) return set_err(c, st, err);
        for (int i = 0; i < n_cohorts; i++)
            if (cohorts[i].status) return set_err(c, cohorts[i].status, "cohort " + std::to_string(i) + " failed");
        return KG_OK;
    });
}

int kg_fp32_peak(int device, double* tflops) {
    if (!tflops) return KG_EINVAL;
    std::string err;
    try {
        return kg::fp32_peak(device, *tflops, err);
    } catch (...) {
        return KG_ECUDA;
    }
}

int kg_last_run_stats(kg_ctx* c, kg_run_stats* s) {
    if (!c || !s) return KG_EINVAL;
    *s = c->last;
    return KG_OK;
}

// The autotuner: the launch shape that gives the fewest device milliseconds
// per pair on a sample of the loaded cohort (the first samples, about 32,768
// pairs, every site), by coordinate descent over three parameters in turn,
// each candidate run twice and timed the second time (the first instantiates
// its graphs):
//   * site-pass blocks per SM: the occupancy limit (5), 4, 3;
//   * the work unit (site chunk) of the pass kernel: 32,768, 65,536, 16,384, 8,192
//     list entries;
//   * pairs in flight (the pair tile of a wave) as a share of the job's pairs:
//     a fifth (the default), a third, an eighth, within 4,096..131,072.
// A candidate is kept only when it beats the current choice by more than 2%,
// so run-to-run noise leaves the defaults.  Slots and blocks per SM leave the
// rows bit for bit the same; the work unit changes how a pass's FP64 partial
// sums are grouped, so rows can move in their last bits.
int kg_autotune(kg_ctx* c, int* slots_out, int* bps_out) {
    if (!c) return KG_EINVAL;
    if (!c->loaded) return set_err(c, KG_EINVAL, "load genotypes first");
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        std::string err;
        st = kg::prepare_cohort(c->cohort, c->cohort.raw.as<uint8_t>(), c->cohort.n_samples,
                                c->cohort.n_sites, c->cohort.n_sites, true,
                                c->af_set ? c->af.data() : nullptr, -1.0, c->stream, err);
        if (st) return set_err(c, st, err);
        c->cohort.ml_nk = 0;   // the sample runs the biallelic sites
        // a sample of about 131,072 pairs: enough waves of full slots that the
        // pass kernel runs as in a large job
        int64_t ns = 2;
        while (ns < c->cohort.n_samples && ns * (ns + 1) / 2 < 131072) ns++;
        const int64_t np = ns * (ns + 1) / 2;
        const int64_t full_pairs = c->cohort.n_samples * (c->cohort.n_samples + 1) / 2;
        if (c->dout.reserve(sizeof(kg_output) * np) != cudaSuccess)
            return set_err(c, KG_ENOMEM, "cannot allocate device output rows");
        kg::PairJob jb;
        jb.panel = &c->cohort;
        jb.n_x = ns;
        jb.d_out = c->dout.as<kg_output>();
        int bps = 0, unit = 0, div = 5;
        // The site-pass shape (blocks per SM, work unit) is judged by the pass
        // phase's device time: every shape runs the same passes, and the wave
        // tail of a sample does not mislead it.  The sample runs with as many
        // pairs in flight as the whole cohort would get by default (up to its
        // own pairs): a wave's task count sets how much a unit's size costs
        // in load balance, so a sample with fewer slots than the real job
        // would favour small units.  The share of pairs in flight only matters
        // for jobs below 5 x 131,072 pairs; it is judged by the sample's whole
        // device time (automatic slots), and only for such a cohort.
        const int64_t job_slots = std::min<int64_t>(131072, std::max<int64_t>(4096, full_pairs / 5));
        auto cost = [&](int b, int u, int d, bool whole, double& ms) -> int {
            kg::RunConfig cfg = run_config(c, 100);
            cfg.slots = whole ? 0 : std::min<int64_t>(job_slots, np);
            cfg.pass_blocks_per_sm = b;
            cfg.unit_elems = u;
            cfg.slot_divisor = d;
            for (int rep = 0; rep < 2; rep++) {
                kg_run_stats stt{};
                int r = kg::run_pairs({jb}, cfg, c->ws, c->stream, stt, err);
                if (r && r != KG_ENOSITES) return r;
                ms = whole ? stt.pair_kernel_ms : stt.pass_ms;
            }
            return KG_OK;
        };
        double best = 0.0;
        st = cost(bps, unit, div, false, best);
        if (st) return set_err(c, st, err);
        auto consider = [&](int b, int u, int d, bool whole) -> int {
            double ms = 0.0;
            int r = cost(b, u, d, whole, ms);
            if (r) return r;
            if (ms < 0.98 * best) {
                best = ms;
                bps = b;
                unit = u;
                div = d;
            }
            return KG_OK;
        };
        for (int b : {4, 3})
            if ((st = consider(b, unit, div, false))) return set_err(c, st, err);
        for (int u : {65536, 16384, 8192})
            if ((st = consider(bps, u, div, false))) return set_err(c, st, err);
        if (full_pairs / 5 < 131072) {
            if ((st = cost(bps, unit, div, true, best))) return set_err(c, st, err);
            for (int d : {3, 8})
                if ((st = consider(bps, unit, d, true))) return set_err(c, st, err);
        }
        c->wave_slots = 0;
        c->pass_bps = bps;
        c->unit_elems = unit;
        c->slot_divisor = div;
        if (slots_out) *slots_out = 0;
        if (bps_out) *bps_out = bps;
        return KG_OK;
    });
}

// ---------------------------------------------------------------- serving

int kg_panel_load(kg_ctx* c, const uint8_t* codes, int64_t n_samples, int64_t n_sites, int64_t row_stride,
                  const double* af, double maf) {
    if (!c) return KG_EINVAL;
    return guarded(c, [&]() -> int {
        int st = use_device(c);
        if (st) return st;
        std::unique_lock<std::mutex> lk(c->mu);
        // wait for in-flight requests before replacing the panel
        c->cv.wait(lk, [&] { return c->in_flight == 0 && c->pending.empty(); });
        std::string err;
        c->panel_ready = false;
        st = kg::prepare_cohort(c->panel, codes, n_samples, n_sites, row_stride, false, af,
                                std::isnan(maf) ? -1.0 : maf, c->stream, err);
        if (st) return set_err(c, st, err);
        c->panel.raw.release();
        c->panel_ready = true;
        c->panel_gen++;
        if (c->workers.empty()) {
            c->workers.resize(kServeWorkers);
            for (auto& w : c->workers)
                if (cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess)
                    return set_err(c, KG_ECUDA, "cannot create the serving streams");
        }
        if (c->servers.empty()) {
            c->stop = false;
            for (int w = 0; w < kServeWorkers; w++) c->servers.emplace_back(serve_loop, c, w);
        }
        return KG_OK;
    });
}

int kg_submit(kg_ctx* c, const uint8_t* query_codes, int64_t n_query, int64_t row_stride,
              const uint8_t* site_mask, uint64_t iterations, int64_t* request_id) {
    if (!c) return KG_EINVAL;
    if (!request_id) return set_err(c, KG_EINVAL, "request_id is NULL");
    return guarded(c, [&]() -> int {
        std::lock_guard<std::mutex> lk(c->mu);
        if (!c->panel_ready) return set_err(c, KG_EINVAL, "no panel loaded");
        const int64_t ns = c->panel.n_sites;
        if (!query_codes || n_query <= 0 || row_stride < ns || iterations == 0)
            return set_err(c, KG_EINVAL, "query rows must be positive and cover the panel's sites");
        auto r = std::make_shared<Request>();
        r->id = c->next_id++;
        r->n_query = n_query;
        r->iterations = iterations;
        r->codes.resize((size_t)(n_query * ns));
        for (int64_t i = 0; i < n_query; i++) {
            const uint8_t* src = query_codes + i * row_stride;
            for (int64_t s = 0; s < ns; s++)
                if (src[s] > 3) return set_err(c, KG_EINVAL, "genotype codes must be 0, 1, 2 or 3 (missing)");
            std::memcpy(r->codes.data() + i * ns, src, (size_t)ns);
        }
        if (site_mask) r->mask.assign(site_mask, site_mask + ns);
        c->requests[r->id] = r;
        c->pending.push_back(r->id);
        *request_id = r->id;
        c->cv.notify_all();
        return KG_OK;
    });
}

int kg_poll(kg_ctx* c, int64_t id, int* done) {
    if (!c || !done) return KG_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = c->requests.find(id);
    if (it == c->requests.end()) return set_err(c, KG_ENOTFOUND, "unknown request");
    *done = it->second->done ? 1 : 0;
    return KG_OK;
}

int kg_wait(kg_ctx* c, int64_t id, int64_t timeout_ms, kg_output* out, int64_t out_cap, int64_t* n_out) {
    if (!c) return KG_EINVAL;
    return guarded(c, [&]() -> int {
        std::unique_lock<std::mutex> lk(c->mu);
        auto it = c->requests.find(id);
        if (it == c->requests.end()) return set_err(c, KG_ENOTFOUND, "unknown request");
        auto r = it->second;
        auto pred = [&] { return r->done; };
        if (timeout_ms < 0) {
            c->cv.wait(lk, pred);
        } else if (!c->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
            return set_err(c, KG_ETIMEOUT, "request still running");
        }
        if (r->cancelled) {
            c->requests.erase(id);
            return set_err(c, KG_ECANCELED, "request was cancelled");
        }
        if (r->status) {
            std::string e = r->err;
            int s = r->status;
            c->requests.erase(id);
            return set_err(c, s, e);
        }
        int64_t np = (int64_t)r->rows.size();
        if (!out || out_cap < np) return set_err(c, KG_EINVAL, "output capacity too small");
        std::memcpy(out, r->rows.data(), sizeof(kg_output) * np);
        if (n_out) *n_out = np;
        c->requests.erase(id);
        return KG_OK;
    });
}

int kg_cancel(kg_ctx* c, int64_t id) {
    if (!c) return KG_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    auto it = c->requests.find(id);
    if (it == c->requests.end()) return set_err(c, KG_ENOTFOUND, "unknown request");
    it->second->cancelled = true;
    auto& pq = c->pending;
    auto pos = std::find(pq.begin(), pq.end(), id);
    if (pos != pq.end()) {
        pq.erase(pos);
        it->second->done = true;
        it->second->status = KG_ECANCELED;
    }
    c->cv.notify_all();
    return KG_OK;
}

int kg_serving_stats(kg_ctx* c, int64_t* requests, int64_t* pairs, int64_t* launches) {
    if (!c) return KG_EINVAL;
    std::lock_guard<std::mutex> lk(c->mu);
    if (requests) *requests = c->served_requests;
    if (pairs) *pairs = c->served_pairs;
    if (launches) *launches = c->served_launches;
    return KG_OK;
}

}  // extern "C"
