// kg_cli.cpp — the reference-compatible command line (src/cli.rs:12-181) on
// top of the C ABI, plus its VCF reader (src/vcf.rs:96-482) for biallelic SNPs.
//
//   kestrel input.vcf[.gz] kinship.tsv [-a estimate|info] [-f GT|GL|PL]
//           [-t threads] [-i iterations] [-m maf] [-s samples]
//
// Every field becomes a hard call per sample and site: GT directly; PL/GL by the
// most likely genotype (the reference's one-hot PL encoding, 0 at the call and
// 255 elsewhere, maps back exactly).  Missing entries become code 3 and are
// dropped per pair, as the reference's NaN likelihood rows are
// (src/vcf.rs:355,397; src/lanevector.rs:99-104).  Only biallelic SNPs are
// estimated; tri- and tetra-allelic SNPs are counted and skipped.
#include "kg_vcf.h"

#include <charconv>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
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
    bool cls = false;  // --estimator cls: the reference's default GT estimator (CLS/Brier)
    int threads = 0;   // VCF reader threads (0 = all)
};

void log_info(const char* fmt, const std::string& a = "") {
    std::fprintf(stderr, "[INFO] ");
    std::fprintf(stderr, fmt, a.c_str());
    std::fprintf(stderr, "\n");
}

int usage(const char* why) {
    std::fprintf(stderr,
                 "error: %s\n\nUsage: kestrel [OPTIONS] <INPUT> <OUTPUT>\n\n"
                 "Arguments:\n  <INPUT>   VCF file with genotypes (GT) or genotype likelihoods (GL, PL)\n"
                 "  <OUTPUT>  Tab-separated file to write the coefficients to\n\n"
                 "Options:\n  -a, --allele-freqs <estimate|info>  [default: estimate]\n"
                 "  -f, --field <GT|GL|PL>              [default: GT]\n"
                 "  -t, --threads <THREADS>             VCF reader threads [default: all]\n"
                 "  -i, --iterations <ITERATIONS>       [default: 100]\n"
                 "  -m, --minimum-allele-frequency <F>\n"
                 "  -s, --samples <N>\n"
                 "  -e, --estimator <ml|cls>            [default: ml; cls = conditional least squares\n"
                 "                                       with the Brier objective, GT only]\n",
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
            if (v == "ml") o.cls = false;
            else if (v == "cls") o.cls = true;
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
    if (o.cls && o.field != 'T') {
        why = "--estimator cls needs hard calls (-f GT)";
        return false;
    }
    return true;
}

// Shortest round-trip decimal in the layout the reference's TSV writer uses
// (decimal notation for 1e-5 <= |v| < 1e16, else d.ddde[-]x; "NaN", "inf").
std::string fmt_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
    std::string s(buf, r.ptr);
    bool neg = false;
    if (s[0] == '-') { neg = true; s.erase(0, 1); }
    size_t e = s.find('e');
    std::string mant = s.substr(0, e);
    int exp10 = std::atoi(s.c_str() + e + 1);
    std::string digits;
    for (char ch : mant) if (ch != '.') digits.push_back(ch);
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    if (v == 0.0) digits = "0";
    int k = (int)digits.size();
    int kk = exp10 + 1;  // value = 0.digits x 10^kk
    std::string out;
    if (v == 0.0) {
        out = "0.0";
    } else if (k <= kk && kk <= 16) {
        out = digits + std::string(kk - k, '0') + ".0";
    } else if (0 < kk && kk <= 16) {
        out = digits.substr(0, kk) + "." + digits.substr(kk);
    } else if (-5 < kk && kk <= 0) {
        out = "0." + std::string(-kk, '0') + digits;
    } else if (k == 1) {
        out = digits + "e" + std::to_string(kk - 1);
    } else {
        out = digits.substr(0, 1) + "." + digits.substr(1) + "e" + std::to_string(kk - 1);
    }
    return neg ? "-" + out : out;
}

}  // namespace

extern "C" int kg_run_cli(int argc, const char* const* argv) {
    auto t0 = std::chrono::steady_clock::now();
    Options o;
    std::string why;
    if (!parse_args(argc, argv, o, why)) return usage(why.c_str());
    log_info("Kestrel %s", kg_version());
    log_info("Parsing VCF \"%s\"", o.input);
    kg::VcfData vcf;
    std::string err;
    if (kg::read_vcf(o.input, o.field, o.af_info, o.threads, vcf, err)) {
        std::fprintf(stderr, "Error: %s\n", err.c_str());
        return 1;
    }
    log_info("Parsed %s total sites", std::to_string(vcf.total));
    log_info("Skipped %s sites that were not SNPs", std::to_string(vcf.not_snp));
    log_info("Skipped %s tri- or tetra-allelic sites (biallelic sites only)", std::to_string(vcf.multi));
    log_info("Found %s di-allelic sites", std::to_string(vcf.n_sites));
    if (vcf.soft)
        log_info("%s likelihood entries were not one-hot; their most likely genotype was used",
                 std::to_string(vcf.soft));
    const std::vector<std::string>& samples = vcf.samples;
    const std::vector<double>& af = vcf.af;
    const int64_t ns = (int64_t)samples.size(), nv = vcf.n_sites;
    if (nv == 0 || ns == 0) {
        std::fprintf(stderr, "Error: Must have at least one site and one sample\n");
        return 1;
    }
    const kg::Bytes& codes = vcf.codes;
    int64_t nsel = o.samples < 0 ? ns : o.samples;
    if (nsel > ns) {
        std::fprintf(stderr, "Error: Requested samples %lld exceeds total samples %lld\n", (long long)nsel, (long long)ns);
        return 1;
    }
    int64_t np = nsel * (nsel + 1) / 2;
    log_info("Calculating Jacquard coefficients for %s pairs", std::to_string(np));
    std::vector<kg_output> out((size_t)np);
    kg_ctx* ctx = nullptr;
    int st = kg_create(&ctx, 0, 0);
    if (st) {
        std::fprintf(stderr, "Error: no usable CUDA device (%d)\n", st);
        return 1;
    }
    st = kg_load_genotypes(ctx, codes.data(), ns, nv, nv);
    if (!st && o.af_info) st = kg_set_allele_frequencies(ctx, af.data());
    int64_t nout = 0;
    if (!st) {
        if (o.cls) st = kg_relatedness_gt(ctx, nsel, o.iterations, out.data(), np, &nout);
        else st = kg_relatedness(ctx, nsel, o.iterations, o.maf, out.data(), np, &nout);
    }
    if (st) {
        std::fprintf(stderr, "Error: %s\n", kg_last_error(ctx));
        kg_destroy(ctx);
        return 1;
    }
    kg_destroy(ctx);
    uint64_t nonconv = 0;
    for (auto& r : out) nonconv += (r.iters >= o.iterations);
    if (nonconv)
        std::fprintf(stderr, "[WARN] No convergence for %llu pairs, max iterations %llu exceeded\n",
                     (unsigned long long)nonconv, (unsigned long long)o.iterations);
    FILE* f = std::fopen(o.output.c_str(), "w");
    if (!f) {
        std::fprintf(stderr, "Error: cannot write %s\n", o.output.c_str());
        return 1;
    }
    std::fprintf(f, "sample1\tsample2\tkinship\tjacquard1\tjacquard2\tjacquard3\tjacquard4\tjacquard5\t"
                    "jacquard6\tjacquard7\tjacquard8\tjacquard9\titerations\tobjective\tcondition\n");
    const double kv[9] = {1.0, 0.0, 0.5, 0.0, 0.5, 0.0, 0.5, 0.25, 0.0};
    std::string rowbuf;
    for (auto& r : out) {
        double kin = 0.0;
        for (int i = 0; i < 9; i++) kin = std::fma(r.jacquard[i], kv[i], kin);
        rowbuf = samples[r.x] + "\t" + samples[r.y] + "\t" + fmt_f64(kin);
        for (int i = 0; i < 9; i++) rowbuf += "\t" + fmt_f64(r.jacquard[i]);
        rowbuf += "\t" + std::to_string(r.iters) + "\t" + fmt_f64(r.obj) + "\t" + fmt_f64(std::log10(r.cond)) + "\n";
        std::fputs(rowbuf.c_str(), f);
    }
    std::fclose(f);
    double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    char wb[64];
    std::snprintf(wb, sizeof wb, "%.2fs", wall);
    log_info("Wall Time %s", wb);
    return 0;
}
