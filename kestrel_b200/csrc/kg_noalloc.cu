// kg_noalloc.cu — kg_relatedness_noalloc: the estimator without any device
// allocation.
//
// Some callers cannot call cudaMalloc: code that runs where the allocator is
// off limits (inside another framework's memory pool or a custom allocator
// that must not be bypassed, or a process whose device memory is fully
// reserved up front).  For them this entry point takes the
// genotypes and the output rows as device buffers the caller already owns and
// keeps every intermediate (allele counts, frequencies, bit-plane genotypes,
// the per-warp shape lists, the work queue and counters) in one file-scope
// __device__ array of kNoAllocBytes, which every GPU that loads the library
// holds until the process exits.
//
// It launches the same preparation kernels and the same persistent pair
// kernel as kg_relatedness, on a fixed grid of kWarps warps, so its rows equal
// those of kg_relatedness on the same input.  The call is synchronous: it
// waits on the caller's stream for the kept-site count and the pair counters
// before it returns.
//
// The array's device address is looked up once per device and kept for the
// life of the process; after a cudaDeviceReset (or anything else that
// recreates the device's primary context) that address is stale, so the entry
// point must not be used across a device reset.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "kestrel_gpu.h"
#include "kg_pair.cuh"

namespace kg {
// Kernels defined in kg_engine.cu.
__global__ void count_kernel(const uint8_t*, int64_t, int64_t, int64_t, int32_t*, int32_t*, int32_t*, int32_t*);
__global__ void freq_kernel(const int32_t*, const int32_t*, const int32_t*, const double*, int64_t, double, uint64_t,
                            double*, double*, uint8_t*, int, int64_t);
__global__ void scan_block_kernel(const uint8_t*, int64_t, int32_t*, int32_t*);
__global__ void scan_sums_kernel(int32_t*, int64_t, int32_t*);
__global__ void compact_kernel(const uint8_t*, const int32_t*, const int32_t*, const double*,
                               const double*, int64_t, int32_t*, float*, double*, double*);
__global__ void pad_kernel(const int32_t*, int64_t, float*, double*, double*);
__global__ void pack_kernel(const uint8_t*, int64_t, int64_t, const int32_t*, const int32_t*,
                            const uint8_t*, uint2*, int64_t);
}  // namespace kg

extern "C" __global__ void jacquard_pair_kernel(kg::PairLaunch L);

namespace {

constexpr size_t kNoAllocBytes = size_t(48) << 20;   // 48 MiB per device
constexpr int64_t kMaxSites = 32768;
constexpr int64_t kMaxSamples = 512;
constexpr int kWarpsPerBlock = 4;
constexpr int kBlocks = 16;
constexpr int kWarps = kWarpsPerBlock * kBlocks;      // 64 warps
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_setup_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch array for the current device, looked up once
// per device (the array's name is only a host-side stand-in).
int scratch_for_device(int dev, unsigned char** out) {
    if (dev < 0 || dev >= kMaxDevices) return KG_EINVAL;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return KG_ECUDA;
        g_scratch_ptr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_ptr[dev]);
    return KG_OK;
}

struct Carve {
    unsigned char* base;
    size_t used = 0;
    template <class T>
    T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + count * sizeof(T);
        return reinterpret_cast<T*>(base + off);
    }
};

// Fills the one-entry cohort table from the kept-site count on the device.
__global__ void noalloc_table_kernel(kg::CohortDev* table, const uint2* planes, int64_t plane_stride,
                                     const float* p32, const double* p64, const double* q64,
                                     const int32_t* nkept, int64_t n_x, kg_output* out) {
    kg::CohortDev d;
    d.planes_x = planes;
    d.planes_y = planes;
    d.plane_stride = plane_stride;
    d.p32 = p32;
    d.p64 = p64;
    d.q64 = q64;
    d.n_sites = nkept[0];
    d.n_units = (nkept[0] + kg::UNIT_SITES - 1) / kg::UNIT_SITES;
    d.kind = kg::COHORT_TRIANGLE;
    d.method = kg::ESTIMATOR_ML;
    d.n_x = n_x;
    d.n_y = 0;
    d.pair_begin = 0;
    d.n_pairs = n_x * (n_x + 1) / 2;
    d.out = out;
    d.max_iter = 0;   // the single-kernel engine takes the limit from its launch
    d.cls_q = nullptr;
    d.cls_cmulti = nullptr;
    d.cls_m = (double)nkept[0];
    d.ml_gr = nullptr;
    d.ml_obs = nullptr;
    d.ml_site = nullptr;
    d.ml_rows = nullptr;
    d.ml_rows32 = nullptr;
    d.ml_nk = 0;
    d.ml_stride = 0;
    *table = d;
}

}  // namespace

extern "C" int kg_relatedness_noalloc(const uint8_t* d_codes, int64_t n_samples, int64_t n_sites,
                                      int64_t row_stride, uint64_t iterations, double maf,
                                      kg_output* d_out, int64_t out_cap, void* stream) {
    if (!d_codes || !d_out || n_samples <= 0 || n_sites <= 0 || row_stride < n_sites || iterations == 0)
        return KG_EINVAL;
    if (n_samples > kMaxSamples || n_sites > kMaxSites) return KG_ENOMEM;
    const int64_t np = n_samples * (n_samples + 1) / 2;
    if (out_cap < np) return KG_EINVAL;
    // an error the caller's thread left pending is the caller's: report it
    // and leave it in place rather than take it for one of this call's launches
    if (cudaPeekAtLastError() != cudaSuccess) return KG_ECUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return KG_ECUDA;
    unsigned char* base = nullptr;
    int st = scratch_for_device(dev, &base);
    if (st) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    const int64_t n_seg = (n_sites + kg::SEG_SITES - 1) / kg::SEG_SITES;
    const int64_t cap = n_seg * kg::SEG_SITES;
    const int64_t plane_stride = n_seg * kg::SEG_WORDS;
    const int64_t nb = (n_sites + 1023) / 1024;
    const int64_t list_cap = kg::align4(n_sites) + 32;
    Carve cv{base};
    int32_t* rc = cv.take<int32_t>(n_sites);
    int32_t* oc = cv.take<int32_t>(n_sites);
    int32_t* hc = cv.take<int32_t>(n_sites);
    uint8_t* keep = cv.take<uint8_t>(n_sites);
    int32_t* kidx = cv.take<int32_t>(n_sites);
    int32_t* bsum = cv.take<int32_t>(nb);
    int32_t* nkept = cv.take<int32_t>(4);
    double* pfull = cv.take<double>(n_sites);
    double* qfull = cv.take<double>(n_sites);
    float* p32 = cv.take<float>(cap);
    double* p64 = cv.take<double>(cap);
    double* q64 = cv.take<double>(cap);
    int32_t* site_of = cv.take<int32_t>(n_sites);
    uint2* planes = cv.take<uint2>(n_samples * plane_stride);
    double* lists = cv.take<double>(kWarps * list_cap);
    unsigned long long* queue = cv.take<unsigned long long>(1);
    kg::RunCounters* counters = cv.take<kg::RunCounters>(1);
    kg::CohortDev* table = cv.take<kg::CohortDev>(1);
    if (cv.used > kNoAllocBytes) return KG_ENOMEM;

    if (!(maf >= 0.0)) maf = 1.0 / (2.0 * (double)n_samples);
    if (maf > 1.0) return KG_EINVAL;
    // the array keeps the previous call's contents: zero what must start at zero
    cudaError_t e = cudaMemsetAsync(nkept, 0, sizeof(int32_t) * 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, sizeof(kg::RunCounters), s);
    if (e != cudaSuccess) return KG_ECUDA;
    const int g256 = (int)((n_sites + 255) / 256);
    kg::count_kernel<<<g256, 256, 0, s>>>(d_codes, n_samples, n_sites, row_stride, rc, oc, hc, nkept);
    kg::freq_kernel<<<g256, 256, 0, s>>>(rc, oc, hc, nullptr, n_sites, maf, iterations, pfull, qfull, keep, 0,
                                         n_samples);
    kg::scan_block_kernel<<<(int)nb, 1024, 0, s>>>(keep, n_sites, kidx, bsum);
    kg::scan_sums_kernel<<<1, 1024, 0, s>>>(bsum, nb, nkept);
    kg::compact_kernel<<<g256, 256, 0, s>>>(keep, kidx, bsum, pfull, qfull, n_sites, site_of, p32, p64, q64);
    kg::pad_kernel<<<(int)((cap + 255) / 256), 256, 0, s>>>(nkept, cap, p32, p64, q64);
    kg::pack_kernel<<<256, 256, 0, s>>>(d_codes, n_samples, row_stride, site_of, nkept, nullptr, planes,
                                        plane_stride);
    noalloc_table_kernel<<<1, 1, 0, s>>>(table, planes, plane_stride, p32, p64, q64, nkept, n_samples, d_out);
    kg::PairLaunch L;
    L.cohorts = table;
    L.n_cohorts = 1;
    L.precision = KG_PREC_FP32C;
    L.total_pairs = np;
    L.queue = queue;
    L.lists = lists;
    L.list_stride = list_cap;
    L.tune = kg::make_tune(iterations);
    L.counters = counters;
    jacquard_pair_kernel<<<kBlocks, kWarpsPerBlock * 32, kWarpsPerBlock * kg::WARP_SMEM, s>>>(L);
    if (cudaGetLastError() != cudaSuccess) return KG_ECUDA;
    int32_t h[4];
    unsigned long long nosite = 0;
    e = cudaMemcpyAsync(h, nkept, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&nosite, &counters->nosite_pairs, sizeof(nosite), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return KG_ECUDA;
    if (h[1]) return KG_EINVAL;          // a code above 3
    if (h[0] == 0 || nosite) return KG_ENOSITES;
    return KG_OK;
}
