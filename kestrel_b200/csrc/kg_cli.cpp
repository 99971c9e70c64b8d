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
#include <zlib.h>

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
                 "  -t, --threads <THREADS>             accepted, unused on the GPU\n"
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

// Line reader over plain or gzip-compressed text.
struct LineReader {
    gzFile f = nullptr;
    std::vector<char> buf;
    explicit LineReader(const std::string& path) { f = gzopen(path.c_str(), "rb"); buf.resize(1 << 20); }
    ~LineReader() { if (f) gzclose(f); }
    bool ok() const { return f != nullptr; }
    bool next(std::string& line) {
        line.clear();
        for (;;) {
            if (!gzgets(f, buf.data(), (int)buf.size())) return !line.empty();
            size_t n = std::strlen(buf.data());
            line.append(buf.data(), n);
            if (n && buf[n - 1] == '\n') {
                line.pop_back();
                if (!line.empty() && line.back() == '\r') line.pop_back();
                return true;
            }
        }
    }
};

void split(const std::string& s, char sep, std::vector<std::string_view>& out) {
    out.clear();
    size_t b = 0;
    for (size_t i = 0; i <= s.size(); i++) {
        if (i == s.size() || s[i] == sep) {
            out.emplace_back(s.data() + b, i - b);
            b = i + 1;
        }
    }
}

void split_sv(std::string_view s, char sep, std::vector<std::string_view>& out) {
    out.clear();
    size_t b = 0;
    for (size_t i = 0; i <= s.size(); i++) {
        if (i == s.size() || s[i] == sep) {
            out.emplace_back(s.data() + b, i - b);
            b = i + 1;
        }
    }
}

bool is_base(std::string_view b) {
    return b.size() == 1 && std::strchr("ACGTacgt", b[0]) != nullptr;
}

// Genotype code of one sample's FORMAT value; false on a malformed entry.
bool parse_call(std::string_view v, char field, uint8_t& code, uint64_t& soft) {
    std::vector<std::string_view> parts;
    if (field == 'T') {
        // alleles separated by / or |
        int a[2];
        int k = 0;
        size_t b = 0;
        bool missing = false;
        for (size_t i = 0; i <= v.size(); i++) {
            if (i == v.size() || v[i] == '/' || v[i] == '|') {
                std::string_view t = v.substr(b, i - b);
                if (k >= 2) return false;
                if (t == ".") {
                    missing = true;
                    a[k++] = 0;
                } else {
                    int x = 0;
                    auto r = std::from_chars(t.data(), t.data() + t.size(), x);
                    if (r.ec != std::errc() || x < 0 || x > 1) return false;
                    a[k++] = x;
                }
                b = i + 1;
            }
        }
        if (missing) { code = 3; return true; }
        if (k != 2) return false;
        code = (uint8_t)(a[0] + a[1]);
        return true;
    }
    split_sv(v, ',', parts);
    if (parts.size() == 1 && parts[0] == ".") { code = 3; return true; }
    if (parts.size() != 3) return false;
    double val[3];
    bool any_missing = false;
    for (int i = 0; i < 3; i++) {
        if (parts[i] == ".") { any_missing = true; val[i] = 0; continue; }
        std::string t(parts[i]);
        char* end = nullptr;
        val[i] = std::strtod(t.c_str(), &end);
        if (end == t.c_str()) return false;
    }
    if (any_missing) { code = 3; return true; }
    // likelihood scale: PL = -10 log10 L, GL = log10 L
    double ll[3];
    for (int i = 0; i < 3; i++) ll[i] = (field == 'P') ? -val[i] / 10.0 : val[i];
    int best = 0;
    for (int i = 1; i < 3; i++) if (ll[i] > ll[best]) best = i;
    for (int i = 0; i < 3; i++)
        if (i != best && ll[best] - ll[i] < 25.5 - 1e-9) { soft++; break; }
    code = (uint8_t)best;
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
    LineReader rd(o.input);
    if (!rd.ok()) {
        std::fprintf(stderr, "Error: cannot open %s\n", o.input.c_str());
        return 1;
    }
    std::string line;
    std::vector<std::string> samples;
    std::vector<std::string_view> cols, fmt;
    std::vector<std::vector<uint8_t>> sites;  // per site, codes per sample
    std::vector<double> af;
    uint64_t total = 0, not_snp = 0, multi = 0, soft = 0;
    const char* key = o.field == 'T' ? "GT" : (o.field == 'P' ? "PL" : "GL");
    while (rd.next(line)) {
        if (line.rfind("##", 0) == 0) continue;
        if (line.rfind("#CHROM", 0) == 0) {
            split(line, '\t', cols);
            for (size_t i = 9; i < cols.size(); i++) samples.emplace_back(cols[i]);
            continue;
        }
        if (line.empty()) continue;
        total++;
        split(line, '\t', cols);
        if (cols.size() < 9 + samples.size() || samples.empty()) {
            std::fprintf(stderr, "Error: malformed record %llu\n", (unsigned long long)total);
            return 1;
        }
        std::vector<std::string_view> alts;
        split_sv(cols[4], ',', alts);
        bool snp = is_base(cols[3]);
        for (auto& a : alts) snp = snp && is_base(a);
        if (!snp) { not_snp++; continue; }
        if (alts.size() != 1) { multi++; continue; }
        split_sv(cols[8], ':', fmt);
        int fi = -1;
        for (size_t i = 0; i < fmt.size(); i++) if (fmt[i] == key) fi = (int)i;
        if (fi < 0) {
            std::fprintf(stderr, "Error: No %s data found\n", key);
            return 1;
        }
        std::vector<uint8_t> row(samples.size());
        std::vector<std::string_view> sub;
        for (size_t s = 0; s < samples.size(); s++) {
            split_sv(cols[9 + s], ':', sub);
            std::string_view v = (fi < (int)sub.size()) ? sub[fi] : std::string_view(".");
            if (!parse_call(v, o.field, row[s], soft)) {
                std::fprintf(stderr, "Error: Value %.*s is not a valid %s\n", (int)v.size(), v.data(), key);
                return 1;
            }
        }
        if (o.af_info) {
            std::vector<std::string_view> info;
            split_sv(cols[7], ';', info);
            double a = NAN;
            for (auto& kv : info)
                if (kv.rfind("AF=", 0) == 0) a = std::strtod(std::string(kv.substr(3)).c_str(), nullptr);
            if (std::isnan(a)) {
                std::fprintf(stderr, "Error: No AF info found\n");
                return 1;
            }
            double alt = std::min(std::max(a, 0.0), 1.0);
            af.push_back(1.0 - alt);
            af.push_back(a);
        }
        sites.push_back(std::move(row));
    }
    log_info("Parsed %s total sites", std::to_string(total));
    log_info("Skipped %s sites that were not SNPs", std::to_string(not_snp));
    log_info("Skipped %s tri- or tetra-allelic sites (biallelic sites only)", std::to_string(multi));
    log_info("Found %s di-allelic sites", std::to_string(sites.size()));
    if (soft) log_info("%s likelihood entries were not one-hot; their most likely genotype was used", std::to_string(soft));
    const int64_t ns = (int64_t)samples.size(), nv = (int64_t)sites.size();
    if (nv == 0 || ns == 0) {
        std::fprintf(stderr, "Error: Must have at least one site and one sample\n");
        return 1;
    }
    std::vector<uint8_t> codes((size_t)(ns * nv));
    for (int64_t v = 0; v < nv; v++)
        for (int64_t s = 0; s < ns; s++) codes[(size_t)(s * nv + v)] = sites[v][s];
    sites.clear();
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
