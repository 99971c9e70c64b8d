// kg_multi.cu — tri- and tetra-allelic sites in the maximum-likelihood
// estimator (the reference's GL/PL path on hard calls).
//
// The reference gives every site its allele frequencies (the per-site SQP of
// src/allele/mod.rs:91-134, maf cut), then drops the alleles whose frequency is
// zero (src/wrapper.rs:237-410, remove_zero_frequencies): a site keeps the
// genotypes made of its remaining alleles, in the VCF order, and goes to the
// bi-, tri- or tetra-allelic group by how many remain; a site with fewer than
// two is discarded.  Each pair's row at a site is sum over genotype pairs of
// GLx GLy m[gx][gy] (src/mixture.rs:9-60, the conditional table of
// src/iis.rs:279-462).  With one-hot likelihoods that is:
//   * the row m[g'x][g'y] of the reduced genotypes when both samples' calls
//     use remaining alleles;
//   * a row of zeros when either call uses a dropped allele (its one-hot mass
//     sat on a genotype that was removed); the site still counts for the pair;
//   * no row when either sample is missing (NaN likelihoods, dropped per
//     pair, src/lanevector.rs:99-104).
//
// Device layout after preparation (kept sites k = 0 .. nk - 1, in site order):
//   ml_site[k]  = {first row of the site's table, G' genotypes}
//   ml_rows     = FP64 rows m[g'x][g'y] (9 values), G' x G' per site
//   ml_rows32   = the same rows in FP32, 12 floats each (three float4)
//   ml_gr[s][k] = sample s's reduced genotype (0 .. G' - 1), ML_ZERO_ROW or
//                 ML_MISSING, rows of ml_stride bytes
//   ml_obs[s][w] = bit k % 32 of word k / 32 set when sample s is called at k
// Sites that keep two alleles stay in this generic form (their rows equal the
// biallelic closed forms up to rounding).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "kg_alleleN.cuh"
#include "kg_engine.h"
#include "kg_pair.cuh"

namespace kg {

#define KG_MULTI_TRY(expr)                                                      \
    do {                                                                        \
        cudaError_t e_ = (expr);                                                \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);           \
            return e_ == cudaErrorMemoryAllocation ? KG_ENOMEM : KG_ECUDA;      \
        }                                                                       \
    } while (0)

namespace {

int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Per loaded site (thread per site): genotype-class counts over the called
// samples, the frequency fit (or the caller's frequencies, used as given), the
// remaining alleles and the reduced index of every original genotype.
__global__ void ml_site_kernel(const uint8_t* __restrict__ mg, const uint8_t* __restrict__ mal,
                               const double* __restrict__ af, int64_t n_samples, int64_t n_multi, double maf,
                               uint64_t iterations, int32_t* __restrict__ keep, int32_t* __restrict__ nrows,
                               uint8_t* __restrict__ remap, double* __restrict__ redf, int32_t* __restrict__ flags) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_multi) return;
    const int na = mal[v];
    keep[v] = 0;
    nrows[v] = 0;
    if (na < 3 || na > 4) {
        atomicOr(&flags[0], 1);
        return;
    }
    const int ng = na * (na + 1) / 2;
    int64_t cnt[MAXG];
    for (int g = 0; g < MAXG; g++) cnt[g] = 0;
    bool bad = false;
    for (int64_t s = 0; s < n_samples; s++) {
        const int g = mg[s * n_multi + v];   // adjacent threads read adjacent sites
        if (g == 255) continue;
        if (g >= ng) {
            bad = true;
            break;
        }
        cnt[g]++;
    }
    if (bad) {
        atomicOr(&flags[0], 1);
        return;
    }
    double f[MAXA];
    if (af) {
        for (int a = 0; a < MAXA; a++) f[a] = a < na ? af[4 * v + a] : 0.0;
    } else {
        AlleleClasses C;
        C.a = na;
        C.n = 0;
        for (int g = 0; g < ng; g++)
            if (cnt[g] > 0) {
                C.cls[C.n] = g;
                C.w[C.n] = (double)cnt[g];
                C.n++;
            }
        allele_fit(C, iterations, maf, f);
    }
    // the remaining alleles, in order (NaN frequencies remove every allele)
    int rank[MAXA], nk = 0;
    for (int a = 0; a < MAXA; a++) rank[a] = -1;
    for (int a = 0; a < na; a++)
        if (f[a] > 0.0) rank[a] = nk++;
    for (int a = 0; a < MAXA; a++) redf[4 * v + a] = 0.0;
    for (int a = 0; a < na; a++)
        if (rank[a] >= 0) redf[4 * v + rank[a]] = f[a];
    for (int g = 0; g < MAXG; g++) {
        uint8_t r = ML_ZERO_ROW;
        if (g < ng) {
            int i, j;
            genotype_alleles(g, i, j);
            if (rank[i] >= 0 && rank[j] >= 0) r = (uint8_t)(rank[j] * (rank[j] + 1) / 2 + rank[i]);
        }
        remap[MAXG * v + g] = r;
    }
    if (nk >= 2) {
        const int gk = nk * (nk + 1) / 2;
        keep[v] = 1;
        nrows[v] = gk * gk;
        atomicAdd(&flags[2 + nk], 1);   // sites left with 2, 3, 4 alleles
    }
}

// Exclusive scan of n int32 values by one block, and their total.
constexpr int SCAN1_THREADS = 1024;
__global__ void __launch_bounds__(SCAN1_THREADS) scan_one_block_kernel(const int32_t* __restrict__ in, int64_t n,
                                                                       int32_t* __restrict__ out,
                                                                       int32_t* __restrict__ total) {
    __shared__ int32_t part[SCAN1_THREADS];
    const int t = threadIdx.x;
    const int64_t chunk = (n + SCAN1_THREADS - 1) / SCAN1_THREADS;
    const int64_t b = t * chunk, e = b + chunk < n ? b + chunk : n;
    int32_t s = 0;
    for (int64_t i = b; i < e; i++) s += in[i];
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < SCAN1_THREADS; o <<= 1) {
        const int32_t add = t >= o ? part[t - o] : 0;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    int32_t run = part[t] - s;
    for (int64_t i = b; i < e; i++) {
        const int32_t x = in[i];
        out[i] = run;
        run += x;
    }
    if (t == SCAN1_THREADS - 1) *total = part[t];
}

// Kept sites in order (thread per loaded site): their table entry, their
// original index and remap row, and their rows m[g'x][g'y] over the remaining
// alleles' frequencies.
__global__ void ml_compact_kernel(const int32_t* __restrict__ keep, const int32_t* __restrict__ kidx,
                                  const int32_t* __restrict__ rbase, const uint8_t* __restrict__ remap,
                                  const double* __restrict__ redf, int64_t n_multi, int2* __restrict__ site,
                                  int32_t* __restrict__ orig, uint8_t* __restrict__ kremap,
                                  double* __restrict__ rows, float* __restrict__ rows32) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_multi || !keep[v]) return;
    const int k = kidx[v];
    const double f0 = redf[4 * v], f1 = redf[4 * v + 1], f2 = redf[4 * v + 2], f3 = redf[4 * v + 3];
    const int na = (f2 > 0.0) ? ((f3 > 0.0) ? 4 : 3) : 2;
    const int gk = na * (na + 1) / 2;
    site[k] = make_int2(rbase[v], gk);
    orig[k] = (int32_t)v;
    for (int g = 0; g < MAXG; g++) kremap[MAXG * k + g] = remap[MAXG * v + g];
    double* R = rows + 9 * (int64_t)rbase[v];
    for (int gx = 0; gx < gk; gx++) {
        int i, j;
        genotype_alleles(gx, i, j);
        for (int gy = 0; gy < gk; gy++) {
            int a, b;
            genotype_alleles(gy, a, b);
            const int64_t row = (int64_t)rbase[v] + gx * gk + gy;
            iis_row(i, j, a, b, f0, f1, f2, f3, R + 9 * (gx * gk + gy));
            for (int e = 0; e < 12; e++) rows32[12 * row + e] = e < 9 ? (float)rows[9 * row + e] : 0.f;
        }
    }
}

// Reduced genotype codes and observed masks (thread per sample and kept site;
// a warp covers 32 consecutive kept sites, one mask word).
__global__ void ml_codes_kernel(const uint8_t* __restrict__ mg, int64_t n_samples, int64_t n_multi,
                                const int32_t* __restrict__ orig, const uint8_t* __restrict__ kremap,
                                const int32_t* __restrict__ nk_dev, int64_t stride, uint8_t* __restrict__ gr,
                                uint32_t* __restrict__ obs) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nk = *nk_dev;
    if (k >= stride) return;   // whole warps: stride is a multiple of 32
    for (int64_t s = blockIdx.y; s < n_samples; s += gridDim.y) {
        uint8_t code = ML_MISSING;
        if (k < nk) {
            const int g = mg[s * n_multi + orig[k]];
            code = g == 255 ? ML_MISSING : kremap[MAXG * k + g];
        }
        gr[s * stride + k] = code;
        const unsigned bits = __ballot_sync(0xffffffffu, code != ML_MISSING);
        if ((threadIdx.x & 31) == 0) obs[s * (stride / 32) + (k >> 5)] = bits;
    }
}

}  // namespace

int prepare_ml_multi(Cohort& c, bool have_af, double maf, uint64_t iterations, cudaStream_t st, std::string& err) {
    c.ml_nk = 0;
    for (int64_t& k : c.ml_by_alleles) k = 0;
    if (c.n_multi <= 0) return KG_OK;
    const int64_t n = c.n_multi, ns = c.n_samples;
    if (!(maf >= 0.0)) maf = 1.0 / (2.0 * (double)ns);
    KG_MULTI_TRY((cudaError_t)c.ml_keep.reserve(sizeof(int32_t) * n));
    KG_MULTI_TRY((cudaError_t)c.ml_nrows.reserve(sizeof(int32_t) * n));
    KG_MULTI_TRY((cudaError_t)c.ml_kidx.reserve(sizeof(int32_t) * n));
    KG_MULTI_TRY((cudaError_t)c.ml_rbase.reserve(sizeof(int32_t) * n));
    KG_MULTI_TRY((cudaError_t)c.ml_remap.reserve((size_t)MAXG * n));
    KG_MULTI_TRY((cudaError_t)c.ml_redf.reserve(sizeof(double) * 4 * n));
    KG_MULTI_TRY((cudaError_t)c.ml_count.reserve(sizeof(int32_t) * 8));
    KG_MULTI_TRY(cudaMemsetAsync(c.ml_count.p, 0, sizeof(int32_t) * 8, st));
    // [0] bad flag, [1] kept sites, [2] rows, [4..6] kept sites left with 2, 3, 4 alleles
    int32_t* cnt = c.ml_count.as<int32_t>();
    ml_site_kernel<<<(unsigned)cdiv(n, 128), 128, 0, st>>>(
        c.mg.as<uint8_t>(), c.malleles.as<uint8_t>(), have_af ? c.maf.as<double>() : nullptr, ns, n, maf, iterations,
        c.ml_keep.as<int32_t>(), c.ml_nrows.as<int32_t>(), c.ml_remap.as<uint8_t>(), c.ml_redf.as<double>(), cnt);
    scan_one_block_kernel<<<1, SCAN1_THREADS, 0, st>>>(c.ml_keep.as<int32_t>(), n, c.ml_kidx.as<int32_t>(), cnt + 1);
    scan_one_block_kernel<<<1, SCAN1_THREADS, 0, st>>>(c.ml_nrows.as<int32_t>(), n, c.ml_rbase.as<int32_t>(),
                                                       cnt + 2);
    KG_MULTI_TRY(cudaGetLastError());
    int32_t h[8];
    KG_MULTI_TRY(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    KG_MULTI_TRY(cudaStreamSynchronize(st));
    if (h[0]) {
        err = "multi-allelic genotype indices must be below the site's genotype count (or 255, missing), "
              "allele counts 3 or 4";
        return KG_EINVAL;
    }
    const int64_t nk = h[1], nrows = h[2];
    for (int k = 0; k < 3; k++) c.ml_by_alleles[k] = h[4 + k];
    if (nk == 0) return KG_OK;
    const int64_t stride = cdiv(nk, 32) * 32;
    KG_MULTI_TRY((cudaError_t)c.ml_site.reserve(sizeof(int2) * nk));
    KG_MULTI_TRY((cudaError_t)c.ml_orig.reserve(sizeof(int32_t) * nk));
    KG_MULTI_TRY((cudaError_t)c.ml_kremap.reserve((size_t)MAXG * nk));
    KG_MULTI_TRY((cudaError_t)c.ml_rows.reserve(sizeof(double) * 9 * nrows));
    KG_MULTI_TRY((cudaError_t)c.ml_rows32.reserve(sizeof(float) * 12 * nrows));
    KG_MULTI_TRY((cudaError_t)c.ml_gr.reserve((size_t)(ns * stride)));
    KG_MULTI_TRY((cudaError_t)c.ml_obs.reserve(sizeof(uint32_t) * ns * (stride / 32)));
    ml_compact_kernel<<<(unsigned)cdiv(n, 128), 128, 0, st>>>(
        c.ml_keep.as<int32_t>(), c.ml_kidx.as<int32_t>(), c.ml_rbase.as<int32_t>(), c.ml_remap.as<uint8_t>(),
        c.ml_redf.as<double>(), n, c.ml_site.as<int2>(), c.ml_orig.as<int32_t>(), c.ml_kremap.as<uint8_t>(),
        c.ml_rows.as<double>(), c.ml_rows32.as<float>());
    const dim3 cg((unsigned)cdiv(stride, 256), (unsigned)std::min<int64_t>(ns, 65535));
    ml_codes_kernel<<<cg, 256, 0, st>>>(c.mg.as<uint8_t>(), ns, n, c.ml_orig.as<int32_t>(), c.ml_kremap.as<uint8_t>(),
                                        cnt + 1, stride, c.ml_gr.as<uint8_t>(), c.ml_obs.as<uint32_t>());
    KG_MULTI_TRY(cudaGetLastError());
    c.ml_nk = nk;
    c.ml_stride = stride;
    return KG_OK;
}

}  // namespace kg
