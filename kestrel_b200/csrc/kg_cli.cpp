// kg_cli.cpp — the reference-compatible command line (src/cli.rs:12-181) on
// top of the C ABI; its VCF reader (src/vcf.rs:96-482) is kg_vcf.cpp.  The CUDA context is created while the VCF is read, and the
// output rows are formatted on the host threads in blocks, written in order.
//
//   kestrel input.vcf[.gz] kinship.tsv [-a estimate|info] [-f GT|GL|PL]
//           [-t threads] [-i iterations] [-m maf] [-s samples]
//
// Every field becomes a hard call per sample and site: GT directly; PL/GL by the
// most likely genotype (the reference's one-hot PL encoding, 0 at the call and
// 255 elsewhere, maps back exactly).  Missing entries become code 3 and are
// dropped per pair, as the reference's NaN likelihood rows are
// (src/vcf.rs:355,397; src/lanevector.rs:99-104).  Tri- and tetra-allelic
// SNPs go to the estimators as genotype indices (kg_load_multiallelic): the
// CLS estimator uses the ones every sample calls, the ML estimator all of them
// (with the reference's frequency cut and drop of zero-frequency alleles).
// Files with soft likelihoods run the soft-likelihood estimator on their
// biallelic SNPs.
#include "kg_threads.h"
#include "kg_vcf.h"

#include <sys/resource.h>
#include <sys/time.h>

#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "kestrel_gpu.h"

namespace {

struct Options {
    std::string input, output;
    bool af_info = false;
    char field = 'T';  // 'T' GT, 'L' GL, 'P' PL
    uint64_t iterations = 100;
    double maf = NAN;
    int64_t samples = -1;
    int estimator = -1;  // -1 unset, 0 ml, 1 cls
    bool cls = false;    // CLS/Brier: the reference's estimator for -f GT, the default there
    int threads = 0;   // host threads for VCF reading and output writing (0 = all)
};

// Log lines in the reference's format (env_logger without timestamp or target,
// src/cli.rs:68-71): the level padded to five characters in brackets.
void log_info(const char* fmt, const std::string& a = "") {
    std::fprintf(stderr, "[INFO ] ");
    std::fprintf(stderr, fmt, a.c_str());
    std::fprintf(stderr, "\n");
}

// A duration as Rust's {:.2?} prints it: seconds above one second, else
// milliseconds, microseconds or nanoseconds, two decimals.
std::string rust_duration(double seconds) {
    char b[64];
    if (seconds >= 1.0) std::snprintf(b, sizeof b, "%.2fs", seconds);
    else if (seconds >= 1e-3) std::snprintf(b, sizeof b, "%.2fms", seconds * 1e3);
    else if (seconds >= 1e-6) std::snprintf(b, sizeof b, "%.2f\u00b5s", seconds * 1e6);
    else std::snprintf(b, sizeof b, "%.2fns", seconds * 1e9);
    return b;
}

// The reference's resource checkpoints (src/util.rs:9-37): wall, user and
// kernel time since the tracker was made, and the peak resident set size, as
// "Wall Time ..., User Time ..., Kernel Time ..., Peak Memory ..." (the peak in
// binary units with two decimals).  The estimator calls make one tracker
// after the VCF is read and check it where the reference's wrappers do
// (src/wrapper.rs:84, :158, :204).
struct ResourceTracker {
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    struct rusage u0 {};
    ResourceTracker() { getrusage(RUSAGE_SELF, &u0); }
    static double tv(const timeval& t) { return (double)t.tv_sec + 1e-6 * (double)t.tv_usec; }
    void checkpoint() const {
        struct rusage u {};
        getrusage(RUSAGE_SELF, &u);
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        const double kib = (double)u.ru_maxrss;   // Linux: kibibytes
        const char* unit[] = {"KiB", "MiB", "GiB", "TiB"};
        double v = kib;
        int k = 0;
        while (v >= 1024.0 && k < 3) { v /= 1024.0; k++; }
        char mem[64];
        std::snprintf(mem, sizeof mem, "%.2f %s", v, unit[k]);
        std::fprintf(stderr, "[INFO ] Wall Time %s, User Time %s, Kernel Time %s, Peak Memory %s\n",
                     rust_duration(wall).c_str(), rust_duration(tv(u.ru_utime) - tv(u0.ru_utime)).c_str(),
                     rust_duration(tv(u.ru_stime) - tv(u0.ru_stime)).c_str(), mem);
    }
};

int usage(const char* why) {
    std::fprintf(stderr,
                 "error: %s\n\nUsage: kestrel [OPTIONS] <INPUT> <OUTPUT>\n\n"
                 "Arguments:\n  <INPUT>   VCF file with genotypes (GT) or genotype likelihoods (GL, PL)\n"
                 "  <OUTPUT>  Tab-separated file to write the coefficients to\n\n"
                 "Options:\n  -a, --allele-freqs <estimate|info>  [default: estimate]\n"
                 "  -f, --field <GT|GL|PL>              [default: GT]\n"
                 "  -t, --threads <THREADS>             Host threads (VCF reading, output) [default: all]\n"
                 "  -i, --iterations <ITERATIONS>       [default: 100]\n"
                 "  -m, --minimum-allele-frequency <F>\n"
                 "  -s, --samples <N>\n"
                 "  -e, --estimator <ml|cls>            [default: cls for GT, ml for GL and PL;\n"
                 "                                       cls = conditional least squares with the\n"
                 "                                       Brier objective, GT only]\n",
                 why);
    return 2;
}

bool parse_args(int argc, const char* const* argv, Options& o, std::string& why) {
    std::vector<std::string> pos;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        auto val = [&](std::string& out) -> bool {
            size_t eq = a.find('=');
            if (a.rfind("--", 0) == 0 && eq != std::string::npos) {
                out = a.substr(eq + 1);
                return true;
            }
            if (i + 1 >= argc) return false;
            out = argv[++i];
            return true;
        };
        auto is = [&](const char* s, const char* l) {
            return a == s || a == l || (a.rfind(std::string(l) + "=", 0) == 0);
        };
        std::string v;
        if (is("-a", "--allele-freqs")) {
            if (!val(v)) { why = "missing value for -a"; return false; }
            if (v == "estimate") o.af_info = false;
            else if (v == "info") o.af_info = true;
            else { why = "invalid value '" + v + "' for --allele-freqs"; return false; }
        } else if (is("-f", "--field")) {
            if (!val(v)) { why = "missing value for -f"; return false; }
            if (v == "GT") o.field = 'T';
            else if (v == "GL") o.field = 'L';
            else if (v == "PL") o.field = 'P';
            else { why = "invalid value '" + v + "' for --field"; return false; }
        } else if (is("-t", "--threads")) {
            if (!val(v) || std::atol(v.c_str()) <= 0) { why = "threads must be a positive integer"; return false; }
            o.threads = (int)std::atol(v.c_str());
        } else if (is("-i", "--iterations")) {
            if (!val(v)) { why = "missing value for -i"; return false; }
            long long n = std::atoll(v.c_str());
            if (n <= 0) { why = "iterations must be a positive integer"; return false; }
            o.iterations = (uint64_t)n;
        } else if (is("-m", "--minimum-allele-frequency")) {
            if (!val(v)) { why = "missing value for -m"; return false; }
            o.maf = std::atof(v.c_str());
        } else if (is("-e", "--estimator")) {
            if (!val(v)) { why = "missing value for -e"; return false; }
            if (v == "ml") o.estimator = 0;
            else if (v == "cls") o.estimator = 1;
            else { why = "invalid value '" + v + "' for --estimator"; return false; }
        } else if (is("-s", "--samples")) {
            if (!val(v)) { why = "missing value for -s"; return false; }
            o.samples = std::atoll(v.c_str());
        } else if (a == "-h" || a == "--help") {
            why = "help";
            return false;
        } else if (!a.empty() && a[0] == '-' && a.size() > 1) {
            why = "unexpected argument '" + a + "'";
            return false;
        } else {
            pos.push_back(a);
        }
    }
    if (pos.size() != 2) {
        why = "expected <INPUT> and <OUTPUT>";
        return false;
    }
    o.input = pos[0];
    o.output = pos[1];
    // the reference runs CLS on GT (src/cli.rs:108-118) and ML on GL/PL
    o.cls = o.estimator < 0 ? o.field == 'T' : o.estimator == 1;
    if (o.cls && o.field != 'T') {
        why = "--estimator cls needs hard calls (-f GT)";
        return false;
    }
    return true;
}

// Shortest round-trip decimal in the layout the reference's TSV writer uses
// (decimal notation for 1e-5 <= |v| < 1e16, else d.ddde[-]x; "NaN", "inf").
// Writes at most 32 characters at out and returns their count.
int fmt_f64(double v, char* out) {
    if (std::isnan(v)) {
        std::memcpy(out, "NaN", 3);
        return 3;
    }
    if (std::isinf(v)) {
        if (v > 0) {
            std::memcpy(out, "inf", 3);
            return 3;
        }
        std::memcpy(out, "-inf", 4);
        return 4;
    }
    char buf[40];
    const auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    const char* p = buf;
    char* o = out;
    if (*p == '-') {
        *o++ = '-';
        p++;
    }
    // the significant digits (no point, no trailing zeros) and the exponent
    char digits[24];
    int k = 0;
    for (; p < r.ptr && *p != 'e'; p++)
        if (*p != '.') digits[k++] = *p;
    int exp10 = 0;
    bool neg_exp = false;
    for (p++; p < r.ptr; p++) {
        if (*p == '-') neg_exp = true;
        else if (*p != '+') exp10 = exp10 * 10 + (*p - '0');
    }
    if (neg_exp) exp10 = -exp10;
    while (k > 1 && digits[k - 1] == '0') k--;
    auto put = [&](const char* x, int n) {
        std::memcpy(o, x, (size_t)n);
        o += n;
    };
    auto zeros = [&](int n) {
        for (int i = 0; i < n; i++) *o++ = '0';
    };
    auto exponent = [&](int x) {
        *o++ = 'e';
        const auto e = std::to_chars(o, o + 8, x);
        o = e.ptr;
    };
    const int kk = exp10 + 1;  // value = 0.digits x 10^kk
    if (v == 0.0) {
        put("0.0", 3);
    } else if (k <= kk && kk <= 16) {
        put(digits, k);
        zeros(kk - k);
        put(".0", 2);
    } else if (0 < kk && kk <= 16) {
        put(digits, kk);
        *o++ = '.';
        put(digits + kk, k - kk);
    } else if (-5 < kk && kk <= 0) {
        put("0.", 2);
        zeros(-kk);
        put(digits, k);
    } else if (k == 1) {
        put(digits, 1);
        exponent(kk - 1);
    } else {
        put(digits, 1);
        *o++ = '.';
        put(digits + 1, k - 1);
        exponent(kk - 1);
    }
    return (int)(o - out);
}

// One TSV row of a pair's result.
void append_row(std::string& dst, const kg_output& r, const std::vector<std::string>& samples) {
    static const double kv[9] = {1.0, 0.0, 0.5, 0.0, 0.5, 0.0, 0.5, 0.25, 0.0};
    double kin = 0.0;
    for (int i = 0; i < 9; i++) kin = std::fma(r.jacquard[i], kv[i], kin);
    char b[32 * 13 + 64];
    char* o = b;
    auto num = [&](double x) {
        *o++ = '\t';
        o += fmt_f64(x, o);
    };
    num(kin);
    for (int i = 0; i < 9; i++) num(r.jacquard[i]);
    *o++ = '\t';
    o = std::to_chars(o, o + 24, r.iters).ptr;
    num(r.obj);
    num(std::log10(r.cond));
    *o++ = '\n';
    dst += samples[r.x];
    dst += '\t';
    dst += samples[r.y];
    dst.append(b, (size_t)(o - b));
}

// The CUDA context (about a second to create) is made on another thread while
// the VCF is read.
struct DeviceInit {
    kg_ctx* ctx = nullptr;
    int st = 0;
    std::thread th;
    DeviceInit() : th([this] { st = kg_create(&ctx, 0, 0); }) {}
    DeviceInit(const DeviceInit&) = delete;
    DeviceInit& operator=(const DeviceInit&) = delete;
    ~DeviceInit() {
        join();
        release();
    }
    void join() {
        if (th.joinable()) th.join();
    }
    void release() {
        if (ctx) kg_destroy(ctx);
        ctx = nullptr;
    }
};

}  // namespace

extern "C" int kg_run_cli(int argc, const char* const* argv) {
    Options o;
    std::string why;
    if (!parse_args(argc, argv, o, why)) return usage(why.c_str());
    log_info("Kestrel %s", kg_version());
    log_info("Parsing VCF \"%s\"", o.input);
    DeviceInit dev;
    kg::VcfData vcf;
    std::string err;
    if (kg::read_vcf(o.input, o.field, o.af_info, o.threads, vcf, err)) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return 1;
    }
    log_info("Parsed %s total sites", std::to_string(vcf.total));
    log_info("Skipped %s sites that were not SNPs", std::to_string(vcf.not_snp));
    if (o.cls) {
        // the CLS estimator uses the sites every sample calls, tri- and
        // tetra-allelic ones included (src/vcf.rs:127-181, :217-221)
        const uint64_t bi_missing = vcf.incomplete - vcf.multi_incomplete;
        log_info("Skipped %s sites with missing data", std::to_string(vcf.incomplete));
        log_info("Found %s di-allelic sites", std::to_string(vcf.n_sites - (int64_t)bi_missing));
        log_info("Found %s tri-allelic sites", std::to_string(vcf.tri_full));
        log_info("Found %s tetra-allelic sites", std::to_string(vcf.tetra_full));
    } else {
        // the GL/PL reader's counts (src/vcf.rs:238-320)
        log_info("Found %s di-allelic sites", std::to_string(vcf.n_sites));
        log_info("Found %s tri-allelic sites", std::to_string(vcf.tri));
        log_info("Found %s tetra-allelic sites", std::to_string(vcf.tetra));
    }
    // GL/PL likelihoods that are not all one-hot go to the soft-likelihood
    // estimator, as the reference's GL path fits them (src/wrapper.rs:89-330)
    const bool soft_path = o.field != 'T' && !vcf.gl.empty();
    if (soft_path) {
        log_info("%s likelihood entries are not one-hot: estimating from the soft likelihoods",
                 std::to_string(vcf.soft + vcf.multi_soft));
        if (o.af_info) {
            std::fprintf(stderr, "Error: allele frequencies from INFO/AF cannot be used with soft likelihoods\n");
            return 1;
        }
    }
    const std::vector<std::string>& samples = vcf.samples;
    const std::vector<double>& af = vcf.af;
    const int64_t ns = (int64_t)samples.size(), nv = vcf.n_sites;
    if (nv == 0 || ns == 0) {
        std::fprintf(stderr, "Error: Must have at least one site and one sample\n");
        return 1;
    }
    int64_t nsel = o.samples < 0 ? ns : o.samples;
    if (nsel > ns) {
        std::fprintf(stderr, "Error: Requested samples %lld exceeds total samples %lld\n", (long long)nsel, (long long)ns);
        return 1;
    }
    int64_t np = nsel * (nsel + 1) / 2;
    log_info("Calculating Jacquard coefficients for %s pairs", std::to_string(np));
    std::vector<kg_output> out((size_t)np);
    dev.join();
    if (dev.st) {
        std::fprintf(stderr, "Error: no usable CUDA device (%d)\n", dev.st);
        return 1;
    }
    kg_ctx* ctx = dev.ctx;
    int st = 0;
    int64_t nout = 0;
    // the estimator's resource tracker starts where the reference's wrapper
    // call does, with the VCF read; the ML path checks it once the inputs are
    // on the device (the reference: after its allele frequencies) and again
    // after the estimate, the CLS path once at the end
    const ResourceTracker tracker;
    if (soft_path) {
        st = kg_load_likelihoods(ctx, vcf.gl.data(), ns, nv);
        // tri- and tetra-allelic records: their likelihoods by allele count
        for (int a = 3; a <= 4 && !st && vcf.n_multi > 0 && !vcf.mgl.empty(); a++) {
            const int ng = a * (a + 1) / 2;
            std::vector<int64_t> sel;
            for (int64_t r = 0; r < vcf.n_multi; r++)
                if (vcf.malleles[(size_t)r] == a) sel.push_back(r);
            if (sel.empty()) continue;
            const int64_t nk = (int64_t)sel.size();
            std::vector<double> g((size_t)(ns * nk * ng));
            for (int64_t s = 0; s < ns; s++)
                for (int64_t k = 0; k < nk; k++)
                    std::memcpy(g.data() + (s * nk + k) * ng,
                                vcf.mgl.data() + ((size_t)s * vcf.n_multi + sel[(size_t)k]) * 10, sizeof(double) * ng);
            st = kg_load_likelihoods_multiallelic(ctx, g.data(), ns, nk, a);
        }
        if (!st) tracker.checkpoint();
        if (!st) st = kg_relatedness_gl(ctx, nsel, o.iterations, o.maf, out.data(), np, &nout);
    } else {
        // the reader's codes go up packed: 2 bits a call plus the observed mask
        std::vector<uint32_t> codes2((size_t)(ns * ((nv + 15) / 16))), observed((size_t)(ns * ((nv + 31) / 32)));
        kg::pack_2bit(vcf, o.threads, codes2.data(), observed.data());
        st = kg_load_genotypes_2bit(ctx, codes2.data(), observed.data(), ns, nv);
        if (!st && o.af_info) st = kg_set_allele_frequencies(ctx, af.data());
        if (!st && vcf.n_multi > 0)
            st = kg_load_multiallelic(ctx, vcf.mcodes.data(), ns, vcf.n_multi, vcf.n_multi, vcf.malleles.data(),
                                      o.af_info ? vcf.maf.data() : nullptr);
        if (!st && !o.cls) tracker.checkpoint();
        if (!st) {
            if (o.cls) st = kg_relatedness_gt(ctx, nsel, o.iterations, out.data(), np, &nout);
            else st = kg_relatedness(ctx, nsel, o.iterations, o.maf, out.data(), np, &nout);
        }
    }
    if (st) {
        std::fprintf(stderr, "Error: %s\n", kg_last_error(ctx));
        return 1;
    }
    if (!o.cls) {
        // the sites the ML estimate used after the frequency cut and the drop
        // of zero-frequency alleles (src/wrapper.rs:321-324; the soft path too)
        kg_run_stats rs{};
        if (kg_last_run_stats(ctx, &rs) == 0) {
            log_info("Identified %s di-allelic sites", std::to_string(rs.sites_used[0]));
            log_info("Identified %s tri-allelic sites", std::to_string(rs.sites_used[1]));
            log_info("Identified %s tetra-allelic sites", std::to_string(rs.sites_used[2]));
            log_info("Discarded %s non-segregating sites", std::to_string(rs.sites_discarded));
        }
    }
    tracker.checkpoint();
    dev.release();
    uint64_t nonconv = 0;
    for (auto& r : out) nonconv += (r.iters >= o.iterations);
    if (nonconv)
        std::fprintf(stderr, "[WARN ] No convergence for %llu pairs, max iterations %llu exceeded\n",
                     (unsigned long long)nonconv, (unsigned long long)o.iterations);
    FILE* f = std::fopen(o.output.c_str(), "w");
    if (!f) {
        std::fprintf(stderr, "Error: cannot write %s\n", o.output.c_str());
        return 1;
    }
    std::fprintf(f, "sample1\tsample2\tkinship\tjacquard1\tjacquard2\tjacquard3\tjacquard4\tjacquard5\t"
                    "jacquard6\tjacquard7\tjacquard8\tjacquard9\titerations\tobjective\tcondition\n");
    // rows formatted in parallel blocks, written in order; a bounded number
    // of rows is held at a time
    const int nt = kg::host_threads(o.threads);
    const int64_t block = 16384;
    std::vector<std::string> text((size_t)nt);
    bool write_failed = false;
    for (int64_t r0 = 0; r0 < nout && !write_failed; r0 += block * nt) {
        const int64_t r1 = std::min<int64_t>(nout, r0 + block * nt);
        // a round with fewer blocks than threads leaves some buffers unused
        for (auto& t : text) t.clear();
        kg::parallel_for(nt, (r1 - r0 + block - 1) / block, [&](int t, int64_t b0, int64_t b1) {
            std::string& dst = text[(size_t)t];
            for (int64_t i = r0 + b0 * block; i < std::min<int64_t>(r1, r0 + b1 * block); i++)
                append_row(dst, out[(size_t)i], samples);
        });
        for (int t = 0; t < nt && !write_failed; t++)
            if (!text[(size_t)t].empty() && std::fwrite(text[(size_t)t].data(), 1, text[(size_t)t].size(), f) != text[(size_t)t].size())
                write_failed = true;
    }
    if (write_failed) {
        std::fclose(f);
        std::fprintf(stderr, "Error: cannot write %s\n", o.output.c_str());
        return 1;
    }
    std::fclose(f);
    return 0;
}
