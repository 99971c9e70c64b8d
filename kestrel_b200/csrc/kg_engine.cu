// kg_engine.cu — device preparation kernels, the persistent pair kernel and
// their host-side launch logic.
//
// Reference behaviour restated here:
//   allele frequencies, count form      src/wrapper.rs:412-428
//   maf zeroing + renormalisation        src/allele/mod.rs:120-126, default maf src/wrapper.rs:101
//   non-segregating site drop            src/wrapper.rs:352-410
//   per-pair driver, start points        src/coefficients.rs:77-136
#include "kg_engine.h"
#include "kg_allele.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "kg_pair.cuh"

namespace kg {

#define KG_CUDA_TRY(expr)                                                       \
    do {                                                                        \
        cudaError_t e_ = (expr);                                                \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);           \
            return e_ == cudaErrorMemoryAllocation ? KG_ENOMEM : KG_ECUDA;      \
        }                                                                       \
    } while (0)

void PinBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
}

int PinBuf::reserve(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    cudaError_t e = cudaHostAlloc(&p, n, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    bytes = n;
    return cudaSuccess;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

int DevBuf::reserve(size_t n) {
    if (n <= bytes && p) return cudaSuccess;
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    bytes = n;
    return cudaSuccess;
}

size_t Cohort::device_bytes() const {
    return raw.bytes + af.bytes + rc.bytes + oc.bytes + hc.bytes + keep.bytes + kidx.bytes + bsum.bytes +
           nkept.bytes + pfull.bytes + qfull.bytes + p32.bytes + p64.bytes + q64.bytes +
           site_of.bytes + planes.bytes + cls_q.bytes + cls_part.bytes + mg.bytes + malleles.bytes + maf.bytes +
           mfreq.bytes + mkeep.bytes + mcount.bytes + mpart.bytes + cmulti.bytes + mgT.bytes + ml_keep.bytes +
           ml_nrows.bytes + ml_kidx.bytes + ml_rbase.bytes + ml_remap.bytes + ml_redf.bytes + ml_count.bytes +
           ml_site.bytes + ml_orig.bytes + ml_kremap.bytes + ml_rows.bytes + ml_rows32.bytes + ml_gr.bytes + ml_obs.bytes;
}

const char* engine_version() { return "kestrel-b200 0.1.0 (sm_100a)"; }

// ------------------------------------------------------------ preparation

constexpr int SCAN_BLOCK = 1024;

// Per raw site: REF allele count, observed samples and heterozygous calls over
// all rows; flags any code above 3.  A thread per site (adjacent threads read
// adjacent bytes of a row).
__global__ void count_kernel(const uint8_t* __restrict__ codes, int64_t n_samples, int64_t n_sites,
                             int64_t stride, int32_t* __restrict__ rc, int32_t* __restrict__ oc,
                             int32_t* __restrict__ hc, int32_t* __restrict__ flags) {
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_sites) return;
    int r = 0, o = 0, h = 0;
    bool bad = false;
    for (int64_t s = 0; s < n_samples; s++) {
        unsigned c = codes[s * stride + v];
        bad |= (c > 3u);
        if (c < 3u) { r += 2 - (int)c; o += 1; h += c == 1u; }
    }
    rc[v] = r;
    oc[v] = o;
    hc[v] = h;
    if (bad) atomicOr(&flags[1], 1);
}

// Frequencies as the ML path sees them and the segregating flag: the
// caller's, or the allele-frequency fit of the reference's GL path on the
// site's genotype-class counts (kg_allele.cuh), capped at `iterations`.
__global__ void freq_kernel(const int32_t* __restrict__ rc, const int32_t* __restrict__ oc,
                            const int32_t* __restrict__ hc, const double* __restrict__ af, int64_t n_sites,
                            double maf, uint64_t iterations, double* __restrict__ pf, double* __restrict__ qf,
                            uint8_t* __restrict__ keep, int cls, int64_t n_samples) {
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_sites) return;
    double x0, x1;
    if (cls) {
        // the CLS estimator's sites: every sample called (the reference's GT
        // reader drops a record with any missing call, src/vcf.rs:217-221);
        // counts over all samples (src/wrapper.rs:412-428), no maf, no drop
        if (af) {
            x0 = af[2 * v];
            x1 = af[2 * v + 1];
        } else {
            const double tot = 2.0 * (double)n_samples;
            x0 = (double)rc[v] / tot;
            x1 = (double)(2 * n_samples - rc[v]) / tot;
        }
        pf[v] = x0;
        qf[v] = x1;
        keep[v] = oc[v] == n_samples ? 1 : 0;
        return;
    }
    if (af) {
        x0 = af[2 * v];
        x1 = af[2 * v + 1];
    } else {
        if (oc[v] == 0) {
            pf[v] = 0.0; qf[v] = 0.0; keep[v] = 0;
            return;
        }
        const int32_t het = hc[v], hom_ref = (rc[v] - het) / 2;
        allele2_frequencies((double)hom_ref, (double)het, (double)(oc[v] - hom_ref - het), iterations, maf, x0, x1);
    }
    pf[v] = x0;
    qf[v] = x1;
    keep[v] = (x0 > 0.0 && x1 > 0.0) ? 1 : 0;
}

__device__ __forceinline__ int warp_incl_scan(int x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    return x;
}

// Block-local exclusive scan of keep flags; block totals to bsum.
__global__ void scan_block_kernel(const uint8_t* __restrict__ keep, int64_t n,
                                  int32_t* __restrict__ kidx, int32_t* __restrict__ bsum) {
    __shared__ int wsum[32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t i = (int64_t)blockIdx.x * SCAN_BLOCK + threadIdx.x;
    int v = (i < n) ? keep[i] : 0;
    int x = warp_incl_scan(v, lane);
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = warp_incl_scan(wsum[lane], lane);
        wsum[lane] = s;
    }
    __syncthreads();
    int pre = (wid > 0 ? wsum[wid - 1] : 0) + x - v;
    if (i < n) kidx[i] = pre;
    if (threadIdx.x == SCAN_BLOCK - 1) bsum[blockIdx.x] = pre + v;
}

// Exclusive scan of the block totals in place (one block); total -> out[0].
__global__ void scan_sums_kernel(int32_t* __restrict__ bsum, int64_t nb, int32_t* __restrict__ out) {
    __shared__ int wsum[32];
    __shared__ int carry;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < nb; base += SCAN_BLOCK) {
        int64_t i = base + threadIdx.x;
        int v = (i < nb) ? bsum[i] : 0;
        int x = warp_incl_scan(v, lane);
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int s = warp_incl_scan(wsum[lane], lane);
            wsum[lane] = s;
        }
        __syncthreads();
        int pre = carry + (wid > 0 ? wsum[wid - 1] : 0) + x - v;
        if (i < nb) bsum[i] = pre;
        __syncthreads();
        if (threadIdx.x == SCAN_BLOCK - 1) carry = pre + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = carry;
}

__global__ void compact_kernel(const uint8_t* __restrict__ keep, const int32_t* __restrict__ kidx,
                               const int32_t* __restrict__ bsum, const double* __restrict__ pf,
                               const double* __restrict__ qf, int64_t n, int32_t* __restrict__ site_of,
                               float* __restrict__ p32, double* __restrict__ p64,
                               double* __restrict__ q64) {
    int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n || !keep[v]) return;
    int64_t k = (int64_t)kidx[v] + bsum[v / SCAN_BLOCK];
    site_of[k] = (int32_t)v;
    p64[freq_index(k)] = pf[v];
    q64[k] = qf[v];
    p32[freq_index(k)] = (float)pf[v];
}

__global__ void pad_kernel(const int32_t* __restrict__ nkept, int64_t cap, float* __restrict__ p32,
                           double* __restrict__ p64, double* __restrict__ q64) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + nkept[0];
    if (k >= cap) return;
    p32[freq_index(k)] = 0.5f;
    p64[freq_index(k)] = 0.5;
    q64[k] = 0.5;
}

// CLS quadratic matrix Q = (1/M) sum over kept sites and all nine (gx, gy) of
// m m^T (src/quadratic.rs:13-37): per-block partial sums of the 45 upper
// entries in a fixed order (deterministic), then one block adds the partials
// in block order.
constexpr int GRAM_BLOCKS = 148;
constexpr int GRAM_THREADS = 128;
__global__ void __launch_bounds__(GRAM_THREADS) cls_gram_kernel(const double* __restrict__ p64,
                                                                const double* __restrict__ q64,
                                                                const int32_t* __restrict__ nkept,
                                                                double* __restrict__ part) {
    __shared__ double sh[45][GRAM_THREADS];
    const int64_t n = nkept[0];
    double h[45];
#pragma unroll
    for (int a = 0; a < 45; a++) h[a] = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * GRAM_THREADS + threadIdx.x; k < n; k += (int64_t)GRAM_BLOCKS * GRAM_THREADS) {
        const double p = p64[freq_index(k)], q = q64[k];
        for (int gx = 0; gx < 3; gx++)
            for (int gy = 0; gy < 3; gy++) {
                double row[9];
                cls_row(gx, gy, p, q, row);
                int a = 0;
#pragma unroll
                for (int i = 0; i < 9; i++)
#pragma unroll
                    for (int j = i; j < 9; j++) h[a++] += row[i] * row[j];
            }
    }
#pragma unroll
    for (int a = 0; a < 45; a++) sh[a][threadIdx.x] = h[a];
    __syncthreads();
    if (threadIdx.x < 45) {
        double s = 0.0;
        for (int t = 0; t < GRAM_THREADS; t++) s += sh[threadIdx.x][t];
        part[(int64_t)blockIdx.x * 45 + threadIdx.x] = s;
    }
}

// Q from the per-block partials of the biallelic sites and, when mpart is not
// NULL, those of the multi-allelic sites after them, divided by the sites used.
__global__ void cls_gram_final_kernel(const double* __restrict__ part, const int32_t* __restrict__ nkept,
                                      const double* __restrict__ mpart, const int32_t* __restrict__ mcount,
                                      double* __restrict__ Q) {
    const int a = threadIdx.x;
    if (a >= 45) return;
    double s = 0.0;
    for (int b = 0; b < GRAM_BLOCKS; b++) s += part[b * 45 + a];
    int64_t m = nkept[0];
    if (mpart) {
        for (int b = 0; b < GRAM_BLOCKS; b++) s += mpart[b * 45 + a];
        m += mcount[0];
    }
    int i = 0, rem = a;
    while (rem >= 9 - i) { rem -= 9 - i; i++; }
    const int j = i + rem;
    const double v = s / (double)m;
    Q[i * 9 + j] = v;
    Q[j * 9 + i] = v;
}

// ---- CLS: tri- and tetra-allelic sites (the reference's gt3 / gt4 of
// src/coefficients.rs:180-224)

// Per site: used when every sample has a call (an index of 255 is missing; the
// scan stops there, as the reader drops such a record), frequencies are allele
// counts / (2 n_samples) (src/wrapper.rs:412-428) or the caller's; an index
// beyond the site's genotypes or an allele count other than 3 or 4 sets the
// bad flag.
__global__ void multi_freq_kernel(const uint8_t* __restrict__ mg, const uint8_t* __restrict__ mal,
                                  const double* __restrict__ maf, int64_t n_samples, int64_t n_multi,
                                  double* __restrict__ mfreq, uint8_t* __restrict__ mkeep,
                                  int32_t* __restrict__ mcount) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_multi) return;
    const int na = mal[v];
    const int ng = na * (na + 1) / 2;
    bool bad = na < 3 || na > 4, complete = true;
    int64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    for (int64_t s = 0; s < n_samples && !bad; s++) {
        const int g = mg[s * n_multi + v];   // adjacent threads read adjacent sites
        if (g == 255) {
            complete = false;
            break;
        }
        if (g >= ng) {
            bad = true;
            break;
        }
        int i, j;
        genotype_alleles(g, i, j);
        c0 += (i == 0) + (j == 0);
        c1 += (i == 1) + (j == 1);
        c2 += (i == 2) + (j == 2);
        c3 += (i == 3) + (j == 3);
    }
    const bool use = complete && !bad;
    const int64_t cnt[4] = {c0, c1, c2, c3};
#pragma unroll
    for (int a = 0; a < 4; a++)
        mfreq[4 * v + a] = !use ? 0.0 : maf ? maf[4 * v + a] : a < na ? (double)cnt[a] / (double)(2 * n_samples) : 0.0;
    mkeep[v] = use ? 1 : 0;
    if (use) atomicAdd(&mcount[0], 1);
    if (bad) atomicOr(&mcount[1], 1);
}

// Per-block partial sums of sum over used sites and all (gx, gy) of m m^T,
// in the layout of cls_gram_kernel.
__global__ void __launch_bounds__(GRAM_THREADS) multi_gram_kernel(const uint8_t* __restrict__ mal,
                                                                  const double* __restrict__ mfreq,
                                                                  const uint8_t* __restrict__ mkeep,
                                                                  int64_t n_multi, double* __restrict__ part) {
    __shared__ double sh[45][GRAM_THREADS];
    double h[45];
#pragma unroll
    for (int a = 0; a < 45; a++) h[a] = 0.0;
    for (int64_t k = (int64_t)blockIdx.x * GRAM_THREADS + threadIdx.x; k < n_multi;
         k += (int64_t)GRAM_BLOCKS * GRAM_THREADS) {
        if (!mkeep[k]) continue;
        const int na = mal[k], ng = na * (na + 1) / 2;
        const double f0 = mfreq[4 * k], f1 = mfreq[4 * k + 1], f2 = mfreq[4 * k + 2], f3 = mfreq[4 * k + 3];
        for (int gx = 0; gx < ng; gx++)
            for (int gy = 0; gy < ng; gy++) {
                int i, j, a1, b1;
                genotype_alleles(gx, i, j);
                genotype_alleles(gy, a1, b1);
                double row[9];
                iis_row(i, j, a1, b1, f0, f1, f2, f3, row);
                int a = 0;
#pragma unroll
                for (int r = 0; r < 9; r++)
#pragma unroll
                    for (int t = r; t < 9; t++) h[a++] += row[r] * row[t];
            }
    }
#pragma unroll
    for (int a = 0; a < 45; a++) sh[a][threadIdx.x] = h[a];
    __syncthreads();
    if (threadIdx.x < 45) {
        double s = 0.0;
        for (int t = 0; t < GRAM_THREADS; t++) s += sh[threadIdx.x][t];
        part[(int64_t)blockIdx.x * 45 + threadIdx.x] = s;
    }
}

// Site-major copy of the genotype indices (out[c * rows + r] = in[r * cols + c])
// through 32 x 32 shared-memory tiles.
__global__ void transpose_u8_kernel(const uint8_t* __restrict__ in, int64_t rows, int64_t cols,
                                    uint8_t* __restrict__ out) {
    __shared__ uint8_t t[32][33];
    const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) t[k][threadIdx.x] = in[r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int64_t c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[c * rows + r] = t[threadIdx.x][k];
    }
}

// Per output row (x, y) of the first ns samples, the 9 sums over used
// multi-allelic sites of m[gx][gy], in site order.  Block per x; per tile of
// MC_SITES sites the block evaluates x's rows m[gx][.] (at most 10 genotypes,
// rows padded to 10 doubles) into shared memory, then each thread adds, for
// its y, the row its genotype selects (y's indices from the site-major copy,
// adjacent threads adjacent samples).
constexpr int MC_SITES = 48;
constexpr int MC_THREADS = 256;
__global__ void __launch_bounds__(MC_THREADS) multi_c_kernel(const uint8_t* __restrict__ mg,
                                                             const uint8_t* __restrict__ mgT,
                                                             const uint8_t* __restrict__ mal,
                                                             const double* __restrict__ mfreq,
                                                             const uint8_t* __restrict__ mkeep, int64_t n_samples,
                                                             int64_t n_multi, int64_t ns, double* __restrict__ cm) {
    __shared__ __align__(16) double tile[MC_SITES * 10 * 10];
    __shared__ uint8_t used[MC_SITES];
    const int64_t x = blockIdx.x;
    const int64_t row0 = x * ns - x * (x - 1) / 2;   // the row of (x, x)
    for (int64_t y0 = x; y0 < ns; y0 += MC_THREADS) {
        const int64_t y = y0 + threadIdx.x;
        double acc[9];
#pragma unroll
        for (int t = 0; t < 9; t++) acc[t] = 0.0;
        for (int64_t v0 = 0; v0 < n_multi; v0 += MC_SITES) {
            const int nv = (int)(n_multi - v0 < MC_SITES ? n_multi - v0 : MC_SITES);
            __syncthreads();   // the previous tile has been read
            for (int e = threadIdx.x; e < nv * 10; e += MC_THREADS) {
                const int vl = e / 10, gy = e - vl * 10;
                const int64_t v = v0 + vl;
                const int na = mal[v], ng = na * (na + 1) / 2;
                const bool use = mkeep[v] != 0;
                if (gy == 0) used[vl] = use ? 1 : 0;
                if (use && gy < ng) {
                    int i, j, k, l;
                    genotype_alleles(mg[x * n_multi + v], i, j);
                    genotype_alleles(gy, k, l);
                    double row[9];
                    iis_row(i, j, k, l, mfreq[4 * v], mfreq[4 * v + 1], mfreq[4 * v + 2], mfreq[4 * v + 3], row);
                    double* dst = tile + (vl * 10 + gy) * 10;
#pragma unroll
                    for (int t = 0; t < 9; t++) dst[t] = row[t];
                }
            }
            __syncthreads();
            if (y < ns) {
                for (int vl = 0; vl < nv; vl++) {
                    if (!used[vl]) continue;   // the same for every thread
                    const int gy = mgT[(v0 + vl) * n_samples + y];
                    const double2* r = reinterpret_cast<const double2*>(tile + (vl * 10 + gy) * 10);
                    const double2 a0 = r[0], a1 = r[1], a2 = r[2], a3 = r[3];
                    const double a8 = tile[(vl * 10 + gy) * 10 + 8];
                    acc[0] += a0.x; acc[1] += a0.y; acc[2] += a1.x; acc[3] += a1.y;
                    acc[4] += a2.x; acc[5] += a2.y; acc[6] += a3.x; acc[7] += a3.y;
                    acc[8] += a8;
                }
            }
        }
        if (y < ns)
#pragma unroll
            for (int t = 0; t < 9; t++) cm[(row0 + (y - x)) * 9 + t] = acc[t];
    }
}

// Warp per (row, 32-site word): lanes fetch the codes of 32 kept sites and two
// ballots build the {lo, hi} planes.  Padding and masked-out sites are 3.
__global__ void pack_kernel(const uint8_t* __restrict__ raw, int64_t n_rows, int64_t stride,
                            const int32_t* __restrict__ site_of, const int32_t* __restrict__ nkept,
                            const uint8_t* __restrict__ mask, uint2* __restrict__ planes,
                            int64_t plane_stride) {
    int lane = threadIdx.x & 31;
    int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nk = nkept[0];
    const int64_t total = n_rows * plane_stride;
    for (int64_t t = warp; t < total; t += nwarps) {
        int64_t row = t / plane_stride;
        int64_t word = t - row * plane_stride;
        int64_t k = word * 32 + lane;
        unsigned c = 3u;
        if (k < nk) {
            int32_t s = site_of[k];
            c = raw[row * stride + s];
            if (mask && !mask[s]) c = 3u;
        }
        unsigned lo = __ballot_sync(0xffffffffu, c & 1u);
        unsigned hi = __ballot_sync(0xffffffffu, (c >> 1) & 1u);
        if (lane == 0) planes[t] = make_uint2(lo, hi);
    }
}

// 2-bit codes (16 per word) + observed mask (32 per word) -> byte codes.
__global__ void unpack_2bit_kernel(const uint32_t* __restrict__ codes2,
                                   const uint32_t* __restrict__ observed, int64_t n_rows,
                                   int64_t n_sites, uint8_t* __restrict__ raw) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total = n_rows * n_sites;
    if (i >= total) return;
    int64_t row = i / n_sites, s = i - row * n_sites;
    int64_t w2 = (n_sites + 15) / 16, wm = (n_sites + 31) / 32;
    unsigned c = (codes2[row * w2 + s / 16] >> (2 * (s % 16))) & 3u;
    bool obs = (observed[row * wm + s / 32] >> (s % 32)) & 1u;
    raw[i] = obs ? (uint8_t)c : (uint8_t)3;
}

static inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

static int grid_for(int64_t n, int threads) { return (int)std::max<int64_t>(1, ceil_div(n, threads)); }

int prepare_cohort(Cohort& c, const uint8_t* codes, int64_t n_samples, int64_t n_sites,
                   int64_t row_stride, bool codes_on_device, const double* af, double maf,
                   cudaStream_t st, std::string& err, bool cls, uint64_t iterations) {
    if (n_samples <= 0 || n_sites <= 0 || row_stride < n_sites) {
        err = "n_samples and n_sites must be positive and row_stride >= n_sites";
        return KG_EINVAL;
    }
    if (n_sites > (int64_t)INT32_MAX || n_samples > (int64_t)INT32_MAX) {
        err = "too many sites or samples";
        return KG_EINVAL;
    }
    c.n_samples = n_samples;
    c.n_sites = n_sites;
    c.n_kept = -1;
    c.cls = cls;
    c.n_seg_max = ceil_div(n_sites, SEG_SITES);
    c.plane_stride = c.n_seg_max * SEG_WORDS;
    const int64_t cap = c.n_seg_max * SEG_SITES;
    const int64_t nb = ceil_div(n_sites, SCAN_BLOCK);
    int64_t stride = row_stride;
    if (!codes_on_device) {
        KG_CUDA_TRY((cudaError_t)c.raw.reserve((size_t)(n_samples * n_sites)));
        if (row_stride == n_sites) {
            KG_CUDA_TRY(cudaMemcpyAsync(c.raw.p, codes, (size_t)(n_samples * n_sites),
                                        cudaMemcpyHostToDevice, st));
        } else {
            KG_CUDA_TRY(cudaMemcpy2DAsync(c.raw.p, (size_t)n_sites, codes, (size_t)row_stride,
                                          (size_t)n_sites, (size_t)n_samples,
                                          cudaMemcpyHostToDevice, st));
        }
        stride = n_sites;
    }
    const uint8_t* draw = codes_on_device ? codes : c.raw.as<uint8_t>();
    KG_CUDA_TRY((cudaError_t)c.rc.reserve(sizeof(int32_t) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.oc.reserve(sizeof(int32_t) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.hc.reserve(sizeof(int32_t) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.keep.reserve((size_t)n_sites));
    KG_CUDA_TRY((cudaError_t)c.kidx.reserve(sizeof(int32_t) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.bsum.reserve(sizeof(int32_t) * nb));
    KG_CUDA_TRY((cudaError_t)c.nkept.reserve(sizeof(int32_t) * 4));
    KG_CUDA_TRY((cudaError_t)c.pfull.reserve(sizeof(double) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.qfull.reserve(sizeof(double) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.p32.reserve(sizeof(float) * cap));
    KG_CUDA_TRY((cudaError_t)c.p64.reserve(sizeof(double) * cap));
    KG_CUDA_TRY((cudaError_t)c.q64.reserve(sizeof(double) * cap));
    KG_CUDA_TRY((cudaError_t)c.site_of.reserve(sizeof(int32_t) * n_sites));
    KG_CUDA_TRY((cudaError_t)c.planes.reserve(sizeof(uint2) * n_samples * c.plane_stride));
    const double* daf = nullptr;
    if (af) {
        KG_CUDA_TRY((cudaError_t)c.af.reserve(sizeof(double) * 2 * n_sites));
        KG_CUDA_TRY(cudaMemcpyAsync(c.af.p, af, sizeof(double) * 2 * n_sites,
                                    cudaMemcpyHostToDevice, st));
        daf = c.af.as<double>();
    }
    if (!(maf >= 0.0)) maf = 1.0 / (2.0 * (double)n_samples);
    KG_CUDA_TRY(cudaMemsetAsync(c.nkept.p, 0, sizeof(int32_t) * 4, st));
    count_kernel<<<grid_for(n_sites, 256), 256, 0, st>>>(draw, n_samples, n_sites, stride,
                                                          c.rc.as<int32_t>(), c.oc.as<int32_t>(),
                                                          c.hc.as<int32_t>(), c.nkept.as<int32_t>());
    freq_kernel<<<grid_for(n_sites, 256), 256, 0, st>>>(c.rc.as<int32_t>(), c.oc.as<int32_t>(),
                                                         c.hc.as<int32_t>(), daf, n_sites, maf, iterations,
                                                         c.pfull.as<double>(),
                                                         c.qfull.as<double>(), c.keep.as<uint8_t>(),
                                                         cls ? 1 : 0, n_samples);
    scan_block_kernel<<<(int)nb, SCAN_BLOCK, 0, st>>>(c.keep.as<uint8_t>(), n_sites,
                                                       c.kidx.as<int32_t>(), c.bsum.as<int32_t>());
    scan_sums_kernel<<<1, SCAN_BLOCK, 0, st>>>(c.bsum.as<int32_t>(), nb, c.nkept.as<int32_t>());
    compact_kernel<<<grid_for(n_sites, 256), 256, 0, st>>>(
        c.keep.as<uint8_t>(), c.kidx.as<int32_t>(), c.bsum.as<int32_t>(), c.pfull.as<double>(),
        c.qfull.as<double>(), n_sites, c.site_of.as<int32_t>(), c.p32.as<float>(),
        c.p64.as<double>(), c.q64.as<double>());
    pad_kernel<<<grid_for(cap, 256), 256, 0, st>>>(c.nkept.as<int32_t>(), cap, c.p32.as<float>(),
                                                    c.p64.as<double>(), c.q64.as<double>());
    {
        int64_t work = n_samples * c.plane_stride;
        int blocks = (int)std::min<int64_t>(ceil_div(work, 8), 148 * 32);
        pack_kernel<<<blocks, 256, 0, st>>>(draw, n_samples, stride, c.site_of.as<int32_t>(),
                                            c.nkept.as<int32_t>(), nullptr, c.planes.as<uint2>(),
                                            c.plane_stride);
    }
    if (cls) {
        KG_CUDA_TRY((cudaError_t)c.cls_part.reserve(sizeof(double) * GRAM_BLOCKS * 45));
        KG_CUDA_TRY((cudaError_t)c.cls_q.reserve(sizeof(double) * 81));
        cls_gram_kernel<<<GRAM_BLOCKS, GRAM_THREADS, 0, st>>>(c.p64.as<double>(), c.q64.as<double>(),
                                                              c.nkept.as<int32_t>(), c.cls_part.as<double>());
        cls_gram_final_kernel<<<1, 64, 0, st>>>(c.cls_part.as<double>(), c.nkept.as<int32_t>(), nullptr,
                                                nullptr, c.cls_q.as<double>());
    }
    KG_CUDA_TRY(cudaGetLastError());
    int32_t h[4];
    KG_CUDA_TRY(cudaMemcpyAsync(h, c.nkept.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    KG_CUDA_TRY(cudaStreamSynchronize(st));
    if (h[1]) {
        err = "genotype codes must be 0, 1, 2 or 3 (missing)";
        return KG_EINVAL;
    }
    c.n_kept = h[0];
    if (c.n_kept == 0) {
        err = cls ? "no site with a call for every sample" : "no segregating site left after allele-frequency filtering";
        return KG_ENOSITES;
    }
    return KG_OK;
}

int unpack_2bit(DevBuf& raw, DevBuf& d2, DevBuf& dm, const uint32_t* codes2, const uint32_t* observed,
                int64_t n_samples, int64_t n_sites, cudaStream_t st, std::string& err) {
    if (!codes2 || !observed || n_samples <= 0 || n_sites <= 0) {
        err = "invalid packed genotype arguments";
        return KG_EINVAL;
    }
    int64_t w2 = ceil_div(n_sites, 16), wm = ceil_div(n_sites, 32);
    KG_CUDA_TRY((cudaError_t)d2.reserve(sizeof(uint32_t) * w2 * n_samples));
    KG_CUDA_TRY((cudaError_t)dm.reserve(sizeof(uint32_t) * wm * n_samples));
    KG_CUDA_TRY((cudaError_t)raw.reserve((size_t)(n_samples * n_sites)));
    KG_CUDA_TRY(cudaMemcpyAsync(d2.p, codes2, sizeof(uint32_t) * w2 * n_samples,
                                cudaMemcpyHostToDevice, st));
    KG_CUDA_TRY(cudaMemcpyAsync(dm.p, observed, sizeof(uint32_t) * wm * n_samples,
                                cudaMemcpyHostToDevice, st));
    unpack_2bit_kernel<<<grid_for(n_samples * n_sites, 256), 256, 0, st>>>(
        d2.as<uint32_t>(), dm.as<uint32_t>(), n_samples, n_sites, raw.as<uint8_t>());
    KG_CUDA_TRY(cudaGetLastError());
    KG_CUDA_TRY(cudaStreamSynchronize(st));
    return KG_OK;
}

int prepare_query(const Cohort& panel, QueryPlanes& q, const uint8_t* codes, int64_t n_rows,
                  int64_t row_stride, const uint8_t* site_mask, cudaStream_t st, std::string& err) {
    if (n_rows <= 0 || row_stride < panel.n_sites || !codes) {
        err = "query rows must be positive and cover the panel's sites";
        return KG_EINVAL;
    }
    const int64_t ns = panel.n_sites;
    q.n_rows = n_rows;
    KG_CUDA_TRY((cudaError_t)q.raw.reserve((size_t)(n_rows * ns)));
    KG_CUDA_TRY(cudaMemcpy2DAsync(q.raw.p, (size_t)ns, codes, (size_t)row_stride, (size_t)ns,
                                  (size_t)n_rows, cudaMemcpyHostToDevice, st));
    const uint8_t* dmask = nullptr;
    if (site_mask) {
        KG_CUDA_TRY((cudaError_t)q.mask.reserve((size_t)ns));
        KG_CUDA_TRY(cudaMemcpyAsync(q.mask.p, site_mask, (size_t)ns, cudaMemcpyHostToDevice, st));
        dmask = q.mask.as<uint8_t>();
    }
    KG_CUDA_TRY((cudaError_t)q.planes.reserve(sizeof(uint2) * n_rows * panel.plane_stride));
    int64_t work = n_rows * panel.plane_stride;
    int blocks = (int)std::min<int64_t>(ceil_div(work, 8), 148 * 32);
    pack_kernel<<<blocks, 256, 0, st>>>(q.raw.as<uint8_t>(), n_rows, ns, panel.site_of.as<int32_t>(),
                                        panel.nkept.as<int32_t>(), dmask, q.planes.as<uint2>(),
                                        panel.plane_stride);
    KG_CUDA_TRY(cudaGetLastError());
    return KG_OK;
}

// ----------------------------------------------------------- pair kernel

__device__ __forceinline__ void decode_triangle(int64_t j, int64_t ns, int64_t& x, int64_t& y) {
    // offset(x) = x*ns - x(x-1)/2 pairs precede row x
    double b = 2.0 * (double)ns + 1.0;
    double disc = b * b - 8.0 * (double)j;
    int64_t xi = (int64_t)floor((b - sqrt(fmax(disc, 0.0))) * 0.5);
    if (xi < 0) xi = 0;
    if (xi > ns - 1) xi = ns - 1;
    auto off = [ns](int64_t r) { return r * ns - r * (r - 1) / 2; };
    while (xi > 0 && off(xi) > j) xi--;
    while (xi + 1 < ns && off(xi + 1) <= j) xi++;
    x = xi;
    y = xi + (j - off(xi));
}

extern "C" __global__ void __launch_bounds__(128, 4)
jacquard_pair_kernel(PairLaunch L) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    char* wsm = smem + wib * WARP_SMEM;
    void* lists = L.lists + gw * L.list_stride;
    unsigned long long c_gh = 0, c_obj = 0, c_f64 = 0, c_f64p = 0, c_sites = 0, c_work = 0,
                       c_nosite = 0, c_nonconv = 0, c_fl32 = 0, c_fl64 = 0;
    unsigned long long c_shape[5] = {0, 0, 0, 0, 0};
    unsigned long long c_cyc[5] = {0, 0, 0, 0, 0};
    for (;;) {
        unsigned long long k = 0;
        if (lane == 0) k = atomicAdd(L.queue, 1ull);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= (unsigned long long)L.total_pairs) break;
        int c = 0;
        while (c + 1 < L.n_cohorts && (int64_t)k >= L.cohorts[c + 1].pair_begin) c++;
        const CohortDev& co = L.cohorts[c];
        const int64_t j = (int64_t)k - co.pair_begin;
        int64_t x, y;
        if (co.kind == COHORT_TRIANGLE) {
            decode_triangle(j, co.n_x, x, y);
        } else {
            x = j / co.n_y;
            y = j - x * co.n_y;
        }
        PairLists pl;
        long long tc0 = clock64();
        count_shapes(co, x, y, lane, pl);
        c_cyc[0] += clock64() - tc0;
        kg_output row;
        row.x = (uint64_t)x;
        row.y = (uint64_t)y;
        if (pl.n == 0) {
            for (int i = 0; i < 9; i++) row.jacquard[i] = CUDART_NAN;
            row.obj = CUDART_NAN;
            row.iters = 0;
            row.cond = CUDART_NAN;
            c_nosite++;
        } else {
            long long ts0 = clock64();
            if (L.precision == 1)
                scatter_shapes<double>(co, x, y, lane, pl, static_cast<double*>(lists), wsm);
            else
                scatter_shapes<float>(co, x, y, lane, pl, static_cast<float*>(lists), wsm);
            c_cyc[1] += clock64() - ts0;
            PairResult res;
            const bool self_pair = (co.kind == COHORT_TRIANGLE) && (x == y);
            solve_pair(co, x, y, pl, lists, self_pair, L.precision, L.tune, lane, wsm, res);
            for (int i = 0; i < 9; i++) row.jacquard[i] = res.x[i];
            row.obj = res.f;
            row.iters = res.iters;
            row.cond = res.cond;
            c_cyc[2] += res.cyc_pass;
            c_cyc[3] += res.cyc_solve;
            c_cyc[4] += res.cyc_stream;
            c_gh += res.gh_passes;
            c_obj += res.obj_passes;
            c_f64 += res.fp64_passes;
            c_f64p += res.escalated ? 1 : 0;
            c_sites += (unsigned long long)pl.n;
            c_work += (unsigned long long)pl.n * (unsigned long long)res.gh_passes;
            c_nonconv += (res.iters >= L.tune.sqp_max_iter) ? 1 : 0;
            const int p32 = res.gh_passes - res.fp64_passes;
#pragma unroll
            for (int s = 0; s < 5; s++) {
                c_shape[s] += (unsigned long long)pl.cnt[s];
                c_fl32 += (unsigned long long)pl.cnt[s] *
                          (unsigned long long)(p32 * flops_fp32_lo(s) + res.diff_passes * flops_diff_extra(s));
                c_fl64 += (unsigned long long)pl.cnt[s] * (unsigned long long)(res.fp64_passes * flops_fp64(s));
            }
        }
        // 14 eight-byte words per row, one per lane
        const uint64_t* src = reinterpret_cast<const uint64_t*>(&row);
        uint64_t* dst = reinterpret_cast<uint64_t*>(co.out + j);
        uint64_t wv = 0;
#pragma unroll
        for (int i = 0; i < 14; i++)
            if (lane == i) wv = src[i];
        if (lane < 14) dst[lane] = wv;
    }
    if (lane == 0) {
        atomicAdd(&L.counters->gh_passes, c_gh);
        atomicAdd(&L.counters->obj_passes, c_obj);
        atomicAdd(&L.counters->fp64_passes, c_f64);
        atomicAdd(&L.counters->fp64_pairs, c_f64p);
        atomicAdd(&L.counters->pair_sites, c_sites);
        atomicAdd(&L.counters->work_units, c_work);
        atomicAdd(&L.counters->nosite_pairs, c_nosite);
        atomicAdd(&L.counters->nonconverged, c_nonconv);
        atomicAdd(&L.counters->flops_fp32, c_fl32);
        atomicAdd(&L.counters->flops_fp64, c_fl64);
        for (int s = 0; s < 5; s++) atomicAdd(&L.counters->shape_sites[s], c_shape[s]);
        for (int s = 0; s < 5; s++) atomicAdd(&L.counters->cycles[s], c_cyc[s]);
    }
}

static_assert(sizeof(kg_output) == 14 * 8, "kg_output must be 112 bytes");

int prepare_multi(Cohort& c, bool have_af, int64_t num_samples, cudaStream_t st, std::string& err) {
    c.n_multi_kept = 0;
    if (c.n_multi <= 0) return KG_OK;
    const int64_t n = c.n_multi, rows = num_samples * (num_samples + 1) / 2;
    KG_CUDA_TRY((cudaError_t)c.mfreq.reserve(sizeof(double) * 4 * n));
    KG_CUDA_TRY((cudaError_t)c.mkeep.reserve((size_t)n));
    KG_CUDA_TRY((cudaError_t)c.mcount.reserve(sizeof(int32_t) * 2));
    KG_CUDA_TRY((cudaError_t)c.mpart.reserve(sizeof(double) * GRAM_BLOCKS * 45));
    KG_CUDA_TRY((cudaError_t)c.cmulti.reserve(sizeof(double) * 9 * rows));
    KG_CUDA_TRY((cudaError_t)c.mgT.reserve((size_t)(n * c.n_samples)));
    KG_CUDA_TRY(cudaMemsetAsync(c.mcount.p, 0, sizeof(int32_t) * 2, st));
    multi_freq_kernel<<<grid_for(n, 256), 256, 0, st>>>(c.mg.as<uint8_t>(), c.malleles.as<uint8_t>(),
                                                         have_af ? c.maf.as<double>() : nullptr, c.n_samples, n,
                                                         c.mfreq.as<double>(), c.mkeep.as<uint8_t>(),
                                                         c.mcount.as<int32_t>());
    multi_gram_kernel<<<GRAM_BLOCKS, GRAM_THREADS, 0, st>>>(c.malleles.as<uint8_t>(), c.mfreq.as<double>(),
                                                            c.mkeep.as<uint8_t>(), n, c.mpart.as<double>());
    cls_gram_final_kernel<<<1, 64, 0, st>>>(c.cls_part.as<double>(), c.nkept.as<int32_t>(), c.mpart.as<double>(),
                                            c.mcount.as<int32_t>(), c.cls_q.as<double>());
    {
        const dim3 tg((unsigned)ceil_div(n, 32), (unsigned)ceil_div(c.n_samples, 32));
        transpose_u8_kernel<<<tg, dim3(32, 8), 0, st>>>(c.mg.as<uint8_t>(), c.n_samples, n, c.mgT.as<uint8_t>());
        multi_c_kernel<<<(unsigned)num_samples, MC_THREADS, 0, st>>>(
            c.mg.as<uint8_t>(), c.mgT.as<uint8_t>(), c.malleles.as<uint8_t>(), c.mfreq.as<double>(),
            c.mkeep.as<uint8_t>(), c.n_samples, n, num_samples, c.cmulti.as<double>());
    }
    KG_CUDA_TRY(cudaGetLastError());
    int32_t h[2];
    KG_CUDA_TRY(cudaMemcpyAsync(h, c.mcount.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    KG_CUDA_TRY(cudaStreamSynchronize(st));
    if (h[1]) {
        err = "multi-allelic genotype indices must be below the site's genotype count (or 255, missing), "
              "allele counts 3 or 4";
        return KG_EINVAL;
    }
    c.n_multi_kept = h[0];
    return KG_OK;
}

CohortDev make_cohort_dev(const PairJob& jb, uint64_t iterations) {
    const Cohort& pn = *jb.panel;
    CohortDev d;
    d.planes_y = pn.planes.as<uint2>();
    d.planes_x = (jb.kind == COHORT_RECT) ? jb.query->planes.as<uint2>() : d.planes_y;
    d.plane_stride = pn.plane_stride;
    d.p32 = pn.p32.as<float>();
    d.p64 = pn.p64.as<double>();
    d.q64 = pn.q64.as<double>();
    d.n_sites = (int32_t)pn.n_kept;
    d.n_units = (int32_t)ceil_div(pn.n_kept, UNIT_SITES);
    d.kind = jb.kind;
    d.method = jb.method;
    d.n_x = jb.n_x;
    d.n_y = jb.n_y;
    d.pair_begin = 0;
    d.n_pairs = jb.n_pairs();
    d.out = jb.d_out;
    d.max_iter = jb.iterations ? jb.iterations : iterations;
    d.cls_q = jb.method == ESTIMATOR_CLS ? pn.cls_q.as<double>() : nullptr;
    const bool multi = jb.method == ESTIMATOR_CLS && pn.n_multi_kept > 0;
    d.cls_cmulti = multi ? pn.cmulti.as<double>() : nullptr;
    d.cls_m = (double)pn.n_kept + (multi ? (double)pn.n_multi_kept : 0.0);
    // the ML path's tri- and tetra-allelic sites (whole cohorts only)
    const bool ml = jb.method == ESTIMATOR_ML && jb.kind == COHORT_TRIANGLE && pn.ml_nk > 0;
    d.ml_gr = ml ? pn.ml_gr.as<uint8_t>() : nullptr;
    d.ml_obs = ml ? pn.ml_obs.as<uint32_t>() : nullptr;
    d.ml_site = ml ? pn.ml_site.as<int2>() : nullptr;
    d.ml_rows = ml ? pn.ml_rows.as<double>() : nullptr;
    d.ml_rows32 = ml ? pn.ml_rows32.as<float4>() : nullptr;
    d.ml_nk = ml ? (int32_t)pn.ml_nk : 0;
    d.ml_stride = ml ? (int32_t)pn.ml_stride : 0;
    return d;
}

int64_t list_capacity(const Cohort& panel) { return align4(panel.n_kept) + 32; }

int run_pairs(const std::vector<PairJob>& jobs, const RunConfig& cfg, Workspace& ws,
              cudaStream_t st, kg_run_stats& stats, std::string& err) {
    std::memset(&stats, 0, sizeof(stats));
    if (jobs.empty()) return KG_OK;
    int dev = 0;
    KG_CUDA_TRY(cudaGetDevice(&dev));
    if (ws.sm_count == 0) KG_CUDA_TRY(cudaDeviceGetAttribute(&ws.sm_count, cudaDevAttrMultiProcessorCount, dev));
    int64_t total_pairs = 0;
    int64_t seg_cap = 1;
    std::vector<CohortDev> table(jobs.size());
    for (size_t i = 0; i < jobs.size(); i++) {
        const PairJob& jb = jobs[i];
        CohortDev& d = table[i];
        d = make_cohort_dev(jb, cfg.iterations);
        d.pair_begin = total_pairs;
        total_pairs += d.n_pairs;
        seg_cap = std::max<int64_t>(seg_cap, list_capacity(*jb.panel));
    }
    if (total_pairs == 0) return KG_OK;
    return run_waves(jobs, cfg, ws, st, stats, err, table, total_pairs, seg_cap);
}

// FFMA throughput probe: 16 independent register chains per thread.
__global__ void fma_peak_kernel(float* out, int iters, float b, float c) {
    float a[16];
#pragma unroll
    for (int k = 0; k < 16; k++) a[k] = (float)(threadIdx.x + k) * 1e-3f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) a[k] = fmaf(a[k], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 16; k++) s += a[k];
    if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

int fp32_peak(int device, double& tflops, std::string& err) {
    KG_CUDA_TRY(cudaSetDevice(device));
    int sm = 0;
    KG_CUDA_TRY(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device));
    DevBuf out;
    KG_CUDA_TRY((cudaError_t)out.reserve(1024 * sizeof(float)));
    const int threads = 256, blocks = sm * 8, iters = 8192;
    cudaEvent_t e0, e1;
    KG_CUDA_TRY(cudaEventCreate(&e0));
    KG_CUDA_TRY(cudaEventCreate(&e1));
    fma_peak_kernel<<<blocks, threads>>>(out.as<float>(), 256, 0.999f, 1e-4f);  // warm-up
    cudaEventRecord(e0);
    fma_peak_kernel<<<blocks, threads>>>(out.as<float>(), iters, 0.999f, 1e-4f);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return KG_ECUDA;
    }
    double flops = 2.0 * 16.0 * (double)iters * (double)threads * (double)blocks;
    tflops = flops / ((double)ms * 1e-3) / 1e12;
    return KG_OK;
}

}  // namespace kg

