// kg_soft.cu — the GL/PL estimator on soft genotype likelihoods, biallelic
// sites (src/wrapper.rs:89-330 with src/mixture.rs:67-140 and
// src/coefficients.rs:40-141): per-site allele frequencies by the HWE SQP on
// the samples' likelihoods, then for every pair the Jacquard SQP on the rows
// L_s = sum over (gx, gy) of GLx(gx) GLy(gy) m(gx, gy) of its sites.
//
// Layout: likelihoods double [sample][site][3] (0/0, 0/1, 1/1; linear scale;
// a NaN marks a missing sample).  First form: a warp per pair, lanes over the
// kept sites, everything in FP64; a lane's 45 Hessian sums live in shared
// memory.  Each pass reads both samples' likelihoods, so this form is bound by
// those reads, not by the arithmetic.
#include <cuda_runtime.h>
#include <math_constants.h>

#include <string>
#include <vector>

#include "kestrel_gpu.h"
#include "kg_allele.cuh"
#include "kg_engine.h"
#include "kg_pair.cuh"
#include "kg_rowsolve.cuh"
#include "kg_solver.cuh"

namespace kg {

#define KG_SOFT_TRY(expr)                                                       \
    do {                                                                        \
        cudaError_t e_ = (expr);                                                \
        if (e_ != cudaSuccess) {                                                \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);           \
            return e_ == cudaErrorMemoryAllocation ? KG_ENOMEM : KG_ECUDA;      \
        }                                                                       \
    } while (0)

// Thread per site: frequencies (REF, ALT) and the keep flag (both non-zero
// after the maf cut).  Adjacent threads read adjacent sites of a sample.
__global__ void soft_freq_kernel(const double* __restrict__ gl, int64_t n_samples, int64_t n_sites, double maf,
                                 uint64_t iterations, double* __restrict__ pf, double* __restrict__ qf,
                                 uint8_t* __restrict__ keep) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n_sites) return;
    int64_t called = 0;
    for (int64_t s = 0; s < n_samples; s++) {
        const double* r = gl + (s * n_sites + v) * 3;
        called += !(isnan(r[0]) || isnan(r[1]) || isnan(r[2]));
    }
    double p = 0.0, q = 0.0;
    if (called) {
        auto l = [&](int64_t s, int g) { return gl[(s * n_sites + v) * 3 + g]; };
        allele2_frequencies_soft(l, n_samples, iterations, maf, p, q);
    }
    pf[v] = p;
    qf[v] = q;
    keep[v] = (p > 0.0 && q > 0.0) ? 1 : 0;
}

constexpr int SOFT_WARPS = 4;

// f, g and this lane's Hessian row at x over the pair's rows (-(1/n) sum log(eps
// + L.x), -(1/n) sum L r, (1/n) sum L L' r^2, r = 1/(eps + L.x)); n = rows
// without a NaN.  hs: the lane's 45 upper-triangle sums in shared memory.
__device__ inline int64_t soft_evaluate(const double* __restrict__ gl, int64_t n_sites, const int32_t* __restrict__ kept,
                                        const double* __restrict__ kp, const double* __restrict__ kq, int64_t nk,
                                        int64_t x, int64_t y, const double* xv, double eps, int lane, double* hs,
                                        PairEval& ev) {
    double f = 0.0, g[9];
#pragma unroll
    for (int i = 0; i < 9; i++) g[i] = 0.0;
    for (int a = 0; a < 45; a++) hs[a * 32 + lane] = 0.0;
    int64_t n = 0;
    for (int64_t k = lane; k < nk; k += 32) {
        const int64_t v = kept[k];
        const double* lx = gl + (x * n_sites + v) * 3;
        const double* ly = gl + (y * n_sites + v) * 3;
        const double ax[3] = {lx[0], lx[1], lx[2]}, ay[3] = {ly[0], ly[1], ly[2]};
        if (isnan(ax[0] + ax[1] + ax[2] + ay[0] + ay[1] + ay[2])) continue;
        const double p = kp[k], q = kq[k];
        double L[9];
#pragma unroll
        for (int i = 0; i < 9; i++) L[i] = 0.0;
#pragma unroll
        for (int gx = 0; gx < 3; gx++)
#pragma unroll
            for (int gy = 0; gy < 3; gy++) {
                const double w = ax[gx] * ay[gy];
                double m[9];
                cls_row(gx, gy, p, q, m);
#pragma unroll
                for (int i = 0; i < 9; i++) L[i] = fma(w, m[i], L[i]);
            }
        double d = eps;
#pragma unroll
        for (int i = 0; i < 9; i++) d = fma(xv[i], L[i], d);
        f += log(d);
        const double r = 1.0 / d;
        double b[9];
#pragma unroll
        for (int i = 0; i < 9; i++) {
            g[i] = fma(L[i], r, g[i]);
            b[i] = L[i] * r;
        }
        int a = 0;
#pragma unroll
        for (int i = 0; i < 9; i++)
#pragma unroll
            for (int j = i; j < 9; j++, a++) hs[a * 32 + lane] = fma(b[i], b[j], hs[a * 32 + lane]);
        n++;
    }
    // warp sums (fixed butterfly order)
    for (int off = 16; off > 0; off >>= 1) {
        f += __shfl_xor_sync(0xffffffffu, f, off);
        n += __shfl_xor_sync(0xffffffffu, n, off);
#pragma unroll
        for (int i = 0; i < 9; i++) g[i] += __shfl_xor_sync(0xffffffffu, g[i], off);
    }
    __syncwarp();
    for (int a = 0; a < 45; a++) {
        double h = hs[a * 32 + lane];
        for (int off = 16; off > 0; off >>= 1) h += __shfl_xor_sync(0xffffffffu, h, off);
        if (lane == 0) hs[a * 32] = h;
    }
    __syncwarp();
    const double dn = (double)n;
    ev.f = -f / dn;
#pragma unroll
    for (int i = 0; i < 9; i++) ev.g[i] = -g[i] / dn;
    // lane i < 9 takes row i of H
#pragma unroll
    for (int j = 0; j < 9; j++) {
        double h = 0.0;
        if (lane < 9) {
            const int i0 = lane < j ? lane : j, j0 = lane < j ? j : lane;
            const int a = i0 * 9 - i0 * (i0 - 1) / 2 + (j0 - i0);
            h = hs[a * 32] / dn;
        }
        ev.Hr[j] = h;
    }
    __syncwarp();
    return n;
}

// Warp per output row of the first ns samples (x-major, y >= x), taken from a
// counter; the Jacquard SQP of src/sqp.rs:49-93 in FP64.
__global__ void __launch_bounds__(SOFT_WARPS * 32, 4) soft_pairs_kernel(
    const double* __restrict__ gl, int64_t n_sites, const int32_t* __restrict__ kept, const double* __restrict__ kp,
    const double* __restrict__ kq, int64_t nk, int64_t ns, int64_t n_rows, uint64_t iterations, kg_output* out,
    unsigned long long* next, int* no_rows) {
    __shared__ double hsm[SOFT_WARPS][45 * 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* hs = hsm[w];
    const Tune tu = make_tune(iterations);
    for (;;) {
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(next, 1ull);
        r = __shfl_sync(0xffffffffu, r, 0);
        if ((int64_t)r >= n_rows) break;
        int64_t lo = 0, hi = ns - 1;
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (mid * ns - mid * (mid - 1) / 2 <= (int64_t)r) lo = mid;
            else hi = mid - 1;
        }
        const int64_t x = lo, y = x + ((int64_t)r - (x * ns - x * (x - 1) / 2));
        double xv[9];
#pragma unroll
        for (int i = 0; i < 9; i++) xv[i] = x == y ? 0.0 : 1.0 / 9.0;
        if (x == y) { xv[0] = 0.5; xv[6] = 0.5; }
        normalise9(xv);
        PairEval ev;
        const int64_t n = soft_evaluate(gl, n_sites, kept, kp, kq, nk, x, y, xv, tu.epsilon, lane, hs, ev);
        kg_output* o = out + r;
        if (n == 0) {
            if (lane == 0) {
                o->x = (uint64_t)x;
                o->y = (uint64_t)y;
                for (int i = 0; i < 9; i++) o->jacquard[i] = 0.0;
                o->obj = CUDART_NAN;
                o->iters = 0;
                o->cond = CUDART_NAN;
                atomicOr(no_rows, 1);
            }
            continue;
        }
        double f = ev.f, g[9], Hr[9];
#pragma unroll
        for (int i = 0; i < 9; i++) { g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
        uint64_t iters = tu.sqp_max_iter;
        double cond = CUDART_NAN;
        for (uint64_t it = 0; it < tu.sqp_max_iter; it++) {
            double resid;
            if (kkt_ok(xv, g, tu.sqp_conv_tol, &resid)) {
                iters = it;
                cond = condition_rows(xv, g, Hr, tu.sqp_conv_tol);
                break;
            }
            double cr = 0.0;
            if (lane < 9) cr = pick9(g, lane) - dot_fma(9, Hr, xv);
            double c[9], yv[9], p[9];
            gather9(cr, c);
            qp_simplex_rows(WarpGrp{FULL_MASK}, Hr, c, xv, tu, lane, yv);
#pragma unroll
            for (int i = 0; i < 9; i++) p[i] = yv[i] - xv[i];
            const double tt = tu.bls_sufficient_decrease * dot_fma(9, g, p);
            double alpha = 1.0, xn[9];
            for (int bls = 0;;) {
#pragma unroll
                for (int i = 0; i < 9; i++) xn[i] = xv[i] + alpha * p[i];
                normalise9(xn);
                soft_evaluate(gl, n_sites, kept, kp, kq, nk, x, y, xn, tu.epsilon, lane, hs, ev);
                const bool accept = ev.f <= f + alpha * tt;
                bls++;
                if (accept || bls == tu.bls_max_iter) break;
                alpha *= tu.bls_step_size_reduce;
            }
#pragma unroll
            for (int i = 0; i < 9; i++) { xv[i] = xn[i]; g[i] = ev.g[i]; Hr[i] = ev.Hr[i]; }
            f = ev.f;
        }
        if (lane == 0) {
            o->x = (uint64_t)x;
            o->y = (uint64_t)y;
            for (int i = 0; i < 9; i++) o->jacquard[i] = xv[i];
            o->obj = f;
            o->iters = iters;
            o->cond = cond;
        }
    }
}

int soft_relatedness(const DevBuf& gl, int64_t n_samples, int64_t n_sites, int64_t ns, uint64_t iterations,
                     double maf, kg_output* d_out, cudaStream_t st, std::string& err, int64_t* n_kept) {
    if (!(maf >= 0.0)) maf = 1.0 / (2.0 * (double)n_samples);
    DevBuf pf, qf, keep, idx, kp, kq, ctr;
    KG_SOFT_TRY((cudaError_t)pf.reserve(sizeof(double) * n_sites));
    KG_SOFT_TRY((cudaError_t)qf.reserve(sizeof(double) * n_sites));
    KG_SOFT_TRY((cudaError_t)keep.reserve((size_t)n_sites));
    soft_freq_kernel<<<(unsigned)((n_sites + 127) / 128), 128, 0, st>>>(gl.as<double>(), n_samples, n_sites, maf,
                                                                        iterations, pf.as<double>(), qf.as<double>(),
                                                                        keep.as<uint8_t>());
    KG_SOFT_TRY(cudaGetLastError());
    // the kept sites, compacted on the host (one small copy each way)
    std::vector<double> hp((size_t)n_sites), hq((size_t)n_sites);
    std::vector<uint8_t> hk((size_t)n_sites);
    KG_SOFT_TRY(cudaMemcpyAsync(hp.data(), pf.p, sizeof(double) * n_sites, cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaMemcpyAsync(hq.data(), qf.p, sizeof(double) * n_sites, cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaMemcpyAsync(hk.data(), keep.p, (size_t)n_sites, cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaStreamSynchronize(st));
    std::vector<int32_t> ki;
    std::vector<double> kpv, kqv;
    for (int64_t v = 0; v < n_sites; v++)
        if (hk[(size_t)v]) {
            ki.push_back((int32_t)v);
            kpv.push_back(hp[(size_t)v]);
            kqv.push_back(hq[(size_t)v]);
        }
    const int64_t nk = (int64_t)ki.size();
    if (n_kept) *n_kept = nk;
    if (nk == 0) {
        err = "no segregating site left after allele-frequency filtering";
        return KG_ENOSITES;
    }
    KG_SOFT_TRY((cudaError_t)idx.reserve(sizeof(int32_t) * nk));
    KG_SOFT_TRY((cudaError_t)kp.reserve(sizeof(double) * nk));
    KG_SOFT_TRY((cudaError_t)kq.reserve(sizeof(double) * nk));
    KG_SOFT_TRY((cudaError_t)ctr.reserve(sizeof(unsigned long long) + sizeof(int)));
    KG_SOFT_TRY(cudaMemcpyAsync(idx.p, ki.data(), sizeof(int32_t) * nk, cudaMemcpyHostToDevice, st));
    KG_SOFT_TRY(cudaMemcpyAsync(kp.p, kpv.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    KG_SOFT_TRY(cudaMemcpyAsync(kq.p, kqv.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, st));
    KG_SOFT_TRY(cudaMemsetAsync(ctr.p, 0, sizeof(unsigned long long) + sizeof(int), st));
    unsigned long long* next = ctr.as<unsigned long long>();
    int* no_rows = reinterpret_cast<int*>(next + 1);
    const int64_t rows = ns * (ns + 1) / 2;
    int dev = 0, sms = 148;
    KG_SOFT_TRY(cudaGetDevice(&dev));
    KG_SOFT_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    soft_pairs_kernel<<<(unsigned)(sms * 4), SOFT_WARPS * 32, 0, st>>>(gl.as<double>(), n_sites, idx.as<int32_t>(),
                                                                      kp.as<double>(), kq.as<double>(), nk, ns, rows,
                                                                      iterations, d_out, next, no_rows);
    KG_SOFT_TRY(cudaGetLastError());
    int h_no_rows = 0;
    KG_SOFT_TRY(cudaMemcpyAsync(&h_no_rows, no_rows, sizeof(int), cudaMemcpyDeviceToHost, st));
    KG_SOFT_TRY(cudaStreamSynchronize(st));
    if (h_no_rows) {
        err = "a pair shares no called segregating site";
        return KG_ENOSITES;
    }
    return KG_OK;
}

}  // namespace kg
