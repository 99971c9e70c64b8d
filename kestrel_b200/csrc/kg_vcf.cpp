// kg_vcf.cpp — multithreaded VCF reader (see kg_vcf.h).
#include "kg_vcf.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <new>
#include <stdexcept>

#include "kestrel_gpu.h"
#include "kg_threads.h"

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string_view>
#include <thread>
#include <utility>

namespace kg {
namespace {

// A file's bytes: a read-only mapping of a regular file (the parse threads
// fault its pages in parallel), else a copy read with stdio.
class FileBytes {
public:
    FileBytes() = default;
    FileBytes(const FileBytes&) = delete;
    FileBytes& operator=(const FileBytes&) = delete;
    ~FileBytes() {
        if (map_) munmap(map_, n_);
    }
    bool open(const std::string& path, std::string& err) {
        const int fd = ::open(path.c_str(), O_RDONLY);
        if (fd < 0) {
            err = "cannot open " + path;
            return false;
        }
        struct stat st {};
        if (fstat(fd, &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) {
            void* m = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m != MAP_FAILED) {
                ::close(fd);
                map_ = m;
                n_ = (size_t)st.st_size;
                p_ = static_cast<const char*>(m);
                return true;
            }
        }
        ::close(fd);
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) {
            err = "cannot open " + path;
            return false;
        }
        char buf[1 << 16];
        size_t got;
        while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) copy_.insert(copy_.end(), buf, buf + got);
        const bool bad = std::ferror(f) != 0;
        std::fclose(f);
        if (bad) {
            err = "cannot read " + path;
            return false;
        }
        p_ = copy_.data();
        n_ = copy_.size();
        return true;
    }
    const char* data() const { return p_; }
    size_t size() const { return n_; }

private:
    void* map_ = nullptr;
    const char* p_ = nullptr;
    size_t n_ = 0;
    std::vector<char> copy_;
};

// The decompressed (or mapped) text of a VCF file.
struct Text {
    FileBytes file;                  // plain text: the file itself
    std::unique_ptr<char[]> bgzf;    // BGZF: blocks inflated in parallel
    std::vector<char> gz;            // plain gzip: one serial stream
    const char* data = nullptr;
    size_t size = 0;
};

// BGZF (RFC 1952 members with a 'BC' extra subfield holding the block size
// minus one): the members' starts and uncompressed sizes, or false if any
// member is not BGZF.
bool bgzf_blocks(const char* b, size_t nb, std::vector<size_t>& start, std::vector<size_t>& clen,
                 std::vector<uint32_t>& isize, std::vector<size_t>& hlen) {
    size_t p = 0;
    while (p < nb) {
        if (p + 18 > nb) return false;
        const uint8_t* h = reinterpret_cast<const uint8_t*>(b + p);
        if (h[0] != 0x1f || h[1] != 0x8b || h[2] != 8 || !(h[3] & 4)) return false;
        const size_t xlen = (size_t)h[10] | ((size_t)h[11] << 8);
        size_t q = p + 12;
        const size_t qe = q + xlen;
        if (qe > nb) return false;
        long bsize = -1;
        while (q + 4 <= qe) {
            const uint8_t* s = reinterpret_cast<const uint8_t*>(b + q);
            const size_t slen = (size_t)s[2] | ((size_t)s[3] << 8);
            if (s[0] == 'B' && s[1] == 'C' && slen == 2 && q + 6 <= qe) bsize = (long)s[4] | ((long)s[5] << 8);
            q += 4 + slen;
        }
        if (bsize < 0) return false;
        const size_t total = (size_t)bsize + 1;
        if (p + total > nb || total < 12 + xlen + 8) return false;
        const uint8_t* t = reinterpret_cast<const uint8_t*>(b + p + total - 4);
        start.push_back(p);
        hlen.push_back(12 + xlen);
        clen.push_back(total - 12 - xlen - 8);
        isize.push_back((uint32_t)t[0] | ((uint32_t)t[1] << 8) | ((uint32_t)t[2] << 16) | ((uint32_t)t[3] << 24));
        p += total;
    }
    return true;
}

bool inflate_raw(const char* src, size_t n, char* dst, size_t dn) {
    char dummy[1];
    z_stream zs{};
    if (inflateInit2(&zs, -15) != Z_OK) return false;
    zs.next_in = reinterpret_cast<Bytef*>(const_cast<char*>(src));
    zs.avail_in = (uInt)n;
    zs.next_out = reinterpret_cast<Bytef*>(dn ? dst : dummy);
    zs.avail_out = (uInt)(dn ? dn : 1);
    const int r = inflate(&zs, Z_FINISH);
    const bool ok = r == Z_STREAM_END && zs.total_out == dn;
    inflateEnd(&zs);
    return ok;
}

bool gunzip_stream(const std::string& path, std::vector<char>& text, std::string& err) {
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    gzbuffer(f, 1 << 20);
    const size_t step = (size_t)16 << 20;
    size_t used = 0;
    for (;;) {
        text.resize(used + step);
        const int r = gzread(f, text.data() + used, (unsigned)step);
        if (r < 0) {
            gzclose(f);
            err = "cannot decompress " + path;
            return false;
        }
        used += (size_t)r;
        if ((size_t)r < step) break;
    }
    text.resize(used);
    gzclose(f);
    return true;
}

// The file's text: plain (mapped), BGZF (blocks inflated in parallel) or
// plain gzip.
bool load_text(const std::string& path, int threads, Text& text, std::string& err) {
    if (!text.file.open(path, err)) return false;
    const char* raw = text.file.data();
    const size_t nraw = text.file.size();
    if (nraw < 2 || (uint8_t)raw[0] != 0x1f || (uint8_t)raw[1] != 0x8b) {
        text.data = raw;
        text.size = nraw;
        return true;
    }
    std::vector<size_t> st, cl, hl;
    std::vector<uint32_t> is;
    if (!bgzf_blocks(raw, nraw, st, cl, is, hl)) {
        if (!gunzip_stream(path, text.gz, err)) return false;
        text.data = text.gz.data();
        text.size = text.gz.size();
        return true;
    }
    std::vector<size_t> off(st.size() + 1, 0);
    for (size_t i = 0; i < st.size(); i++) off[i + 1] = off[i] + is[i];
    text.bgzf.reset(new char[std::max<size_t>(1, off.back())]);
    char* out = text.bgzf.get();
    std::vector<char> bad((size_t)std::max(1, threads), 0);
    parallel_for(threads, (int64_t)st.size(), [&](int t, int64_t b, int64_t e) {
        for (int64_t i = b; i < e; i++)
            if (!inflate_raw(raw + st[i] + hl[i], cl[i], out + off[i], is[i])) bad[t] = 1;
    });
    if (std::find(bad.begin(), bad.end(), 1) != bad.end()) {
        err = "cannot decompress " + path;
        return false;
    }
    text.data = out;
    text.size = off.back();
    return true;
}

bool is_base(std::string_view b) { return b.size() == 1 && std::strchr("ACGTacgt", b[0]) != nullptr; }

// Genotype code of one sample's value of the FORMAT key; false if malformed.
// GL/PL: like (when not NULL) gets the call's linear-scale likelihoods as the
// reference's reader makes them (src/vcf.rs:325-420): 10^(GL - max GL) with GL
// read at single precision, or 10^(-PL/10); NaN when the call is missing.
bool parse_call(std::string_view v, char field, uint8_t& code, uint64_t& soft, double* like = nullptr) {
    if (field == 'T') {
        int a[2] = {0, 0};
        int k = 0;
        size_t b = 0;
        bool missing = false;
        for (size_t i = 0; i <= v.size(); i++) {
            if (i == v.size() || v[i] == '/' || v[i] == '|') {
                const std::string_view t = v.substr(b, i - b);
                if (k >= 2) return false;
                if (t == ".") {
                    missing = true;
                    a[k++] = 0;
                } else {
                    int x = 0;
                    const auto r = std::from_chars(t.data(), t.data() + t.size(), x);
                    if (r.ec != std::errc() || r.ptr != t.data() + t.size() || x < 0 || x > 1) return false;
                    a[k++] = x;
                }
                b = i + 1;
            }
        }
        if (missing) {
            code = 3;
            return true;
        }
        if (k != 2) return false;
        code = (uint8_t)(a[0] + a[1]);
        return true;
    }
    if (like) like[0] = like[1] = like[2] = NAN;
    if (v == ".") {
        code = 3;
        return true;
    }
    double val[3];
    int k = 0;
    bool any_missing = false;
    size_t b = 0;
    for (size_t i = 0; i <= v.size(); i++) {
        if (i == v.size() || v[i] == ',') {
            if (k >= 3) return false;
            const std::string_view t = v.substr(b, i - b);
            if (t == ".") {
                any_missing = true;
                val[k++] = 0.0;
            } else {
                const auto r = std::from_chars(t.data(), t.data() + t.size(), val[k]);
                if (r.ec != std::errc() || r.ptr == t.data()) return false;
                k++;
            }
            b = i + 1;
        }
    }
    if (k != 3) return false;
    if (any_missing) {
        code = 3;
        return true;
    }
    if (like) {
        if (field == 'P') {
            for (int i = 0; i < 3; i++) like[i] = std::pow(10.0, -val[i] / 10.0);
        } else {
            double g[3], mx = -INFINITY;
            for (int i = 0; i < 3; i++) {
                g[i] = (double)(float)val[i];
                mx = std::max(mx, g[i]);
            }
            for (int i = 0; i < 3; i++) like[i] = std::pow(10.0, g[i] - mx);
        }
    }
    // likelihood scale: PL = -10 log10 L, GL = log10 L
    double ll[3];
    for (int i = 0; i < 3; i++) ll[i] = (field == 'P') ? -val[i] / 10.0 : val[i];
    int best = 0;
    for (int i = 1; i < 3; i++)
        if (ll[i] > ll[best]) best = i;
    for (int i = 0; i < 3; i++)
        if (i != best && ll[best] - ll[i] < 25.5 - 1e-9) {
            soft++;
            break;
        }
    code = (uint8_t)best;
    return true;
}

// Most likely genotype (VCF order) of a GL/PL value of ng likelihoods at a
// tri- or tetra-allelic site, 255 when the value or an entry is missing; the
// row counts as soft as in parse_call.  like (optional, ng values): the
// linear-scale likelihoods as the reference's reader makes them (NaN when
// missing).  False when the value is not ng numbers.
bool parse_like_index(std::string_view v, char field, int ng, uint8_t& g, uint64_t& soft, double* like = nullptr) {
    if (like)
        for (int i = 0; i < ng; i++) like[i] = NAN;
    if (v == ".") {
        g = 255;
        return true;
    }
    double ll[10], raw[10];
    int k = 0;
    bool any_missing = false;
    size_t b = 0;
    for (size_t i = 0; i <= v.size(); i++) {
        if (i == v.size() || v[i] == ',') {
            if (k >= ng) return false;
            const std::string_view t = v.substr(b, i - b);
            if (t == ".") {
                any_missing = true;
                ll[k++] = 0.0;
            } else {
                double x = 0.0;
                const auto r = std::from_chars(t.data(), t.data() + t.size(), x);
                if (r.ec != std::errc() || r.ptr == t.data()) return false;
                raw[k] = x;
                ll[k++] = field == 'P' ? -x / 10.0 : x;   // PL = -10 log10 L, GL = log10 L
            }
            b = i + 1;
        }
    }
    if (k != ng) return false;
    if (any_missing) {
        g = 255;
        return true;
    }
    if (like) {
        // 10^(-PL/10); 10^(GL - max GL) with GL read at single precision
        // (src/vcf.rs:325-420)
        if (field == 'P') {
            for (int i = 0; i < ng; i++) like[i] = std::pow(10.0, -raw[i] / 10.0);
        } else {
            double mx = -INFINITY, gv[10];
            for (int i = 0; i < ng; i++) {
                gv[i] = (double)(float)raw[i];
                mx = std::max(mx, gv[i]);
            }
            for (int i = 0; i < ng; i++) like[i] = std::pow(10.0, gv[i] - mx);
        }
    }
    int best = 0;
    for (int i = 1; i < ng; i++)
        if (ll[i] > ll[best]) best = i;
    for (int i = 0; i < ng; i++)
        if (i != best && ll[best] - ll[i] < 25.5 - 1e-9) {
            soft++;
            break;
        }
    g = (uint8_t)best;
    return true;
}

// Genotype index (VCF order, j (j + 1) / 2 + i for alleles i <= j) of a GT
// value at a site with n_alleles alleles; 255 when an allele is missing.
// False when the value is not a diploid call of the site's alleles.
bool parse_gt_index(std::string_view v, int n_alleles, uint8_t& g) {
    int a[2] = {0, 0};
    int k = 0;
    size_t b = 0;
    bool missing = false;
    for (size_t i = 0; i <= v.size(); i++) {
        if (i == v.size() || v[i] == '/' || v[i] == '|') {
            const std::string_view t = v.substr(b, i - b);
            if (k >= 2) return false;
            if (t == ".") {
                missing = true;
                a[k++] = 0;
            } else {
                int x = 0;
                const auto r = std::from_chars(t.data(), t.data() + t.size(), x);
                if (r.ec != std::errc() || r.ptr != t.data() + t.size() || x < 0 || x >= n_alleles) return false;
                a[k++] = x;
            }
            b = i + 1;
        }
    }
    if (missing) {
        g = 255;
        return true;
    }
    if (k != 2) return false;
    const int lo = std::min(a[0], a[1]), hi = std::max(a[0], a[1]);
    g = (uint8_t)(hi * (hi + 1) / 2 + lo);
    return true;
}

// Allele digit of a three-character GT value: 0, 1, 2 for '.', -1 otherwise.
struct AlleleTable {
    int8_t a[256];
    constexpr AlleleTable() : a{} {
        for (int i = 0; i < 256; i++) a[i] = -1;
        a[(unsigned char)'0'] = 0;
        a[(unsigned char)'1'] = 1;
        a[(unsigned char)'.'] = 2;
    }
};
constexpr AlleleTable kAllele{};

// Code of "a/b" or "a|b" with a, b in {0, 1, .}; -1 when the value has another
// form (parse_call then decides).  Same results as parse_call on these values.
inline int gt3_code(const char* s) {
    const int a = kAllele.a[(unsigned char)s[0]], b = kAllele.a[(unsigned char)s[2]];
    if ((a | b) < 0 || (s[1] != '/' && s[1] != '|')) return -1;
    return (a == 2 || b == 2) ? 3 : a + b;
}

// 8 x 8 byte transpose: byte j of r[i] moves to byte i of r[j] (three rounds
// of block swaps: 4 x 4, 2 x 2, 1 x 1).
inline void transpose8x8(uint64_t r[8]) {
    for (int i = 0; i < 4; i++) {
        const uint64_t t = ((r[i] >> 32) ^ r[i + 4]) & 0x00000000FFFFFFFFull;
        r[i] ^= t << 32;
        r[i + 4] ^= t;
    }
    for (int i : {0, 1, 4, 5}) {
        const uint64_t t = ((r[i] >> 16) ^ r[i + 2]) & 0x0000FFFF0000FFFFull;
        r[i] ^= t << 16;
        r[i + 2] ^= t;
    }
    for (int i : {0, 2, 4, 6}) {
        const uint64_t t = ((r[i] >> 8) ^ r[i + 1]) & 0x00FF00FF00FF00FFull;
        r[i] ^= t << 8;
        r[i + 1] ^= t;
    }
}

struct Chunk {
    const char* b = nullptr;
    const char* e = nullptr;
    std::vector<uint8_t> rows;   // kept records x samples
    std::vector<double> lrows;   // GL/PL: kept records x samples x 3 linear-scale likelihoods
    std::vector<double> af;
    uint64_t total = 0, not_snp = 0, multi = 0, soft = 0, incomplete = 0;
    int64_t kept = 0;
    // tri- and tetra-allelic records (255 = a missing call)
    std::vector<uint8_t> mrows;  // kept records x samples, genotype indices
    std::vector<uint8_t> malleles;
    std::vector<double> maf;     // 4 per record
    int64_t mkept = 0;
    uint64_t tri = 0, tetra = 0, tri_full = 0, tetra_full = 0, mincomplete = 0;
    uint64_t multi_dropped = 0;  // GT records with a malformed call after a missing one
    uint64_t msoft = 0;          // GL/PL rows of these records that are not one-hot
    std::vector<double> mlrows;  // with likelihoods kept: records x samples x 10 (G used, NaN after)
    bool failed = false;
    uint64_t fail_rec = 0;       // 1-based record index within the chunk
    std::string fail_kind;       // message with %R for the global record number
};

void parse_chunk(Chunk& c, char field, bool af_info, size_t n_samples, bool want_like) {
    const std::string_view key = field == 'T' ? "GT" : (field == 'P' ? "PL" : "GL");
    std::string_view last_fmt;
    int last_fi = -1;
    const char* p = c.b;
    auto fail = [&](const std::string& what) {
        c.failed = true;
        c.fail_rec = c.total;
        c.fail_kind = what;
    };
    while (p < c.e) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(c.e - p)));
        const char* le = nl ? nl : c.e;
        const char* next = nl ? nl + 1 : c.e;
        if (le > p && le[-1] == '\r') le--;
        if (le == p || *p == '#') {
            p = next;
            continue;
        }
        c.total++;
        // the record must have 9 + n_samples columns (extra ones are ignored)
        const size_t tabs = (size_t)std::count(p, le, '\t');
        if (n_samples == 0 || tabs + 1 < 9 + n_samples) {
            fail("malformed record %R");
            return;
        }
        const char* col[10];
        col[0] = p;
        const char* q = p;
        for (int k = 1; k < 10; k++) {
            const char* t = static_cast<const char*>(std::memchr(q, '\t', (size_t)(le - q)));
            q = t + 1;
            col[k] = q;
        }
        auto field_of = [&](int k) { return std::string_view(col[k], (size_t)(col[k + 1] - 1 - col[k])); };
        const std::string_view ref = field_of(3), alt = field_of(4);
        bool snp = is_base(ref);
        size_t n_alts = 0, ab = 0;
        for (size_t i = 0; i <= alt.size(); i++) {
            if (i == alt.size() || alt[i] == ',') {
                snp = snp && is_base(alt.substr(ab, i - ab));
                n_alts++;
                ab = i + 1;
            }
        }
        // REF and every ALT one base; more than four bases is not a SNP
        // (src/vcf.rs:424-444 with the arms of :127-165)
        const int n_bases = 1 + (int)n_alts;
        if (!snp || n_bases > 4) {
            c.not_snp++;
            p = next;
            continue;
        }
        const bool multi = n_bases > 2;
        if (multi) c.multi++;
        const std::string_view fmt = field_of(8);
        int fi = -1;
        if (fmt == last_fmt) {
            fi = last_fi;
        } else {
            size_t fb = 0;
            int idx = 0;
            for (size_t i = 0; i <= fmt.size(); i++) {
                if (i == fmt.size() || fmt[i] == ':') {
                    if (fmt.substr(fb, i - fb) == key) fi = idx;
                    idx++;
                    fb = i + 1;
                }
            }
            last_fmt = fmt;
            last_fi = fi;
        }
        if (fi < 0) {
            fail("No " + std::string(key) + " data found");
            return;
        }
        // the fi-th ':' subfield of the sample starting at s ("." when the
        // value has fewer); s moves to the next sample
        auto sample_value = [&](const char*& s) {
            const char* t = static_cast<const char*>(std::memchr(s, '\t', (size_t)(le - s)));
            const char* se = t ? t : le;
            const char* a = s;
            int idx = 0;
            while (idx < fi) {
                const char* cpos = static_cast<const char*>(std::memchr(a, ':', (size_t)(se - a)));
                if (!cpos) break;
                a = cpos + 1;
                idx++;
            }
            std::string_view v(".");
            if (idx == fi) {
                const char* cpos = static_cast<const char*>(std::memchr(a, ':', (size_t)(se - a)));
                v = std::string_view(a, (size_t)((cpos ? cpos : se) - a));
            }
            s = t ? t + 1 : le;
            return v;
        };
        if (multi) {
            // genotype indices (GT) or the most likely genotype (GL/PL); a
            // missing call is 255.  The CLS estimator leaves out a record with
            // a missing call, as the reference's GT reader does
            // (src/vcf.rs:196-236: it stops at the first missing call, so a bad
            // value after one is not an error there, and the record is
            // dropped here); the ML estimator drops it for that sample's pairs.
            const size_t mb = c.mrows.size();
            c.mrows.resize(mb + n_samples);
            const char* s = col[9];
            const int ng = n_bases * (n_bases + 1) / 2;
            bool missing = false, bad_after_missing = false;
            for (size_t k = 0; k < n_samples; k++) {
                const std::string_view v = sample_value(s);
                uint8_t g = 0;
                double* like = nullptr;
                if (want_like && field != 'T') {
                    if (k == 0) c.mlrows.resize(c.mlrows.size() + n_samples * 10, (double)NAN);
                    like = c.mlrows.data() + c.mlrows.size() - (n_samples - k) * 10;
                }
                const bool ok = field == 'T' ? parse_gt_index(v, n_bases, g)
                                             : parse_like_index(v, field, ng, g, c.msoft, like);
                if (!ok) {
                    if (field == 'T' && missing) {
                        bad_after_missing = true;
                        break;
                    }
                    fail("Value " + std::string(v) + " is not a valid " + std::string(key));
                    return;
                }
                missing = missing || g == 255;
                c.mrows[mb + k] = g;
            }
            if (missing) {
                c.incomplete++;
                c.mincomplete++;
            }
            if (bad_after_missing) {
                c.mrows.resize(mb);
                c.multi_dropped++;
                p = next;
                continue;
            }
            if (af_info) {
                // INFO/AF: one value per ALT; REF = 1 - clamp(sum) (src/vcf.rs:446-482)
                const std::string_view info = field_of(7);
                std::string_view list;
                bool found = false;
                size_t ib = 0;
                for (size_t i = 0; i <= info.size(); i++) {
                    if (i == info.size() || info[i] == ';') {
                        const std::string_view kv = info.substr(ib, i - ib);
                        if (kv.size() >= 3 && kv.substr(0, 3) == "AF=") {
                            list = kv.substr(3);
                            found = true;
                        }
                        ib = i + 1;
                    }
                }
                if (!found) {
                    fail("No AF info found");
                    return;
                }
                double f[4] = {0.0, 0.0, 0.0, 0.0};
                int n_af = 1;
                double alt_sum = 0.0;
                size_t lb = 0;
                for (size_t i = 0; i <= list.size(); i++) {
                    if (i == list.size() || list[i] == ',') {
                        if (n_af >= n_bases) {
                            fail("Too many allele frequencies!");
                            return;
                        }
                        const std::string num(list.substr(lb, i - lb));
                        f[n_af] = std::strtod(num.c_str(), nullptr);
                        alt_sum += f[n_af];
                        n_af++;
                        lb = i + 1;
                    }
                }
                if (n_af != n_bases) {
                    fail("Not enough allele frequencies!");
                    return;
                }
                f[0] = 1.0 - std::min(std::max(alt_sum, 0.0), 1.0);
                c.maf.insert(c.maf.end(), f, f + 4);
            }
            c.malleles.push_back((uint8_t)n_bases);
            if (n_bases == 3) {
                c.tri++;
                if (!missing) c.tri_full++;
            } else {
                c.tetra++;
                if (!missing) c.tetra_full++;
            }
            c.mkept++;
            p = next;
            continue;
        }
        const size_t base = c.rows.size();
        if (base == 0) {
            // room for the chunk's records at this record's length
            const size_t per = (size_t)(next - p);
            c.rows.reserve(((size_t)(c.e - p) / per + 1) * n_samples);
        }
        c.rows.resize(base + n_samples);
        const char* s = col[9];
        const bool gt_first = field == 'T' && fi == 0;
        for (size_t k = 0; k < n_samples; k++) {
            if (gt_first && le - s >= 3) {
                // the common "a/b" call, alone or first of its subfields
                const int code = gt3_code(s);
                const char* after = s + 3;
                if (code >= 0 && (after == le || *after == '\t' || *after == ':')) {
                    c.rows[base + k] = (uint8_t)code;
                    if (after == le) {
                        s = le;
                    } else if (*after == '\t') {
                        s = after + 1;
                    } else {
                        const char* t = static_cast<const char*>(std::memchr(after, '\t', (size_t)(le - after)));
                        s = t ? t + 1 : le;
                    }
                    continue;
                }
            }
            const std::string_view v = sample_value(s);
            double* like = nullptr;
            if (want_like) {
                if (k == 0) c.lrows.resize((base + n_samples) * 3);
                like = c.lrows.data() + (base + k) * 3;
            }
            if (!parse_call(v, field, c.rows[base + k], c.soft, like)) {
                fail("Value " + std::string(v) + " is not a valid " + std::string(key));
                return;
            }
        }
        if (std::memchr(c.rows.data() + base, 3, n_samples)) c.incomplete++;
        if (af_info) {
            const std::string_view info = field_of(7);
            double a = NAN;
            size_t ib = 0;
            for (size_t i = 0; i <= info.size(); i++) {
                if (i == info.size() || info[i] == ';') {
                    const std::string_view kv = info.substr(ib, i - ib);
                    if (kv.size() >= 3 && kv.substr(0, 3) == "AF=") {
                        const std::string num(kv.substr(3));
                        a = std::strtod(num.c_str(), nullptr);
                    }
                    ib = i + 1;
                }
            }
            if (std::isnan(a)) {
                fail("No AF info found");
                return;
            }
            const double altf = std::min(std::max(a, 0.0), 1.0);
            c.af.push_back(1.0 - altf);
            c.af.push_back(a);
        }
        c.kept++;
        p = next;
    }
}

// Sample-major codes[s * nv + v] from the chunks' record-major rows (rows_of(c)
// gives a chunk's rows and record count; records in chunk order): each thread
// a range of samples (a multiple of 8), 8 x 8 tiles of records x samples
// transposed in 64-bit words.
template <class RowsOf>
void transpose_chunks(int threads, size_t ns, int64_t nv, uint8_t* codes, const std::vector<Chunk>& chunks,
                      RowsOf rows_of) {
    const int n_chunks = (int)chunks.size();
    std::vector<int64_t> first((size_t)n_chunks + 1, 0);
    for (int i = 0; i < n_chunks; i++) first[i + 1] = first[i] + rows_of(chunks[i]).second;
    const int64_t n_groups = ((int64_t)ns + 7) / 8;
    parallel_for(threads, n_groups, [&](int, int64_t g0, int64_t g1) {
        const int64_t s0 = g0 * 8, s1 = std::min<int64_t>((int64_t)ns, g1 * 8);
        for (int i = 0; i < n_chunks; i++) {
            const auto rc = rows_of(chunks[i]);
            const uint8_t* rows = rc.first;
            const int64_t kept = rc.second;
            for (int64_t b0 = 0; b0 < kept; b0 += 64) {
                const int64_t b1 = std::min<int64_t>(kept, b0 + 64);
                for (int64_t s = s0; s < s1; s += 8) {
                    int64_t v = b0;
                    if (s + 8 <= s1) {
                        for (; v + 8 <= b1; v += 8) {
                            uint64_t r[8];
                            for (int k = 0; k < 8; k++) std::memcpy(&r[k], rows + (v + k) * (int64_t)ns + s, 8);
                            transpose8x8(r);
                            for (int k = 0; k < 8; k++) std::memcpy(codes + (s + k) * nv + first[i] + v, &r[k], 8);
                        }
                    }
                    for (int64_t t = s; t < std::min<int64_t>(s1, s + 8); t++)
                        for (int64_t w = v; w < b1; w++) codes[t * nv + first[i] + w] = rows[w * (int64_t)ns + t];
                }
            }
        }
    });
}

}  // namespace

int read_vcf(const std::string& path, char field, bool af_info, int threads, VcfData& out, std::string& err) {
    threads = host_threads(threads);
    Text text;
    if (!load_text(path, threads, text, err)) return 1;
    const char* b = text.data;
    const char* e = b + text.size;
    // header: ## lines, then #CHROM with the sample names
    const char* p = b;
    out = VcfData{};
    while (p < e && *p == '#') {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', (size_t)(e - p)));
        const char* le = nl ? nl : e;
        const char* lt = (le > p && le[-1] == '\r') ? le - 1 : le;
        if ((size_t)(lt - p) >= 6 && std::memcmp(p, "#CHROM", 6) == 0) {
            int k = 0;
            const char* f = p;
            for (;;) {
                const char* t = static_cast<const char*>(std::memchr(f, '\t', (size_t)(lt - f)));
                const char* fe = t ? t : lt;
                if (k >= 9) out.samples.emplace_back(f, (size_t)(fe - f));
                k++;
                if (!t) break;
                f = t + 1;
            }
        }
        p = nl ? nl + 1 : e;
    }
    // the body, cut at line boundaries into about 4 chunks per thread
    const int64_t body = (int64_t)(e - p);
    const int n_chunks = body > (1 << 20) ? std::max(1, threads * 4) : 1;
    std::vector<Chunk> chunks((size_t)n_chunks);
    const char* cur = p;
    for (int i = 0; i < n_chunks; i++) {
        const char* target = (i == n_chunks - 1) ? e : p + body * (i + 1) / n_chunks;
        if (target < cur) target = cur;
        if (target < e) {
            const char* nl = static_cast<const char*>(std::memchr(target, '\n', (size_t)(e - target)));
            target = nl ? nl + 1 : e;
        }
        chunks[i].b = cur;
        chunks[i].e = target;
        cur = target;
    }
    const size_t ns = out.samples.size();
    parallel_for(threads, n_chunks, [&](int, int64_t cb, int64_t ce) {
        for (int64_t i = cb; i < ce; i++) parse_chunk(chunks[i], field, af_info, ns, false);
    });
    // a soft GL/PL row: parse again keeping the likelihoods (one-hot files
    // never hold them)
    if (field != 'T') {
        bool any_soft = false, any_failed = false;
        for (auto& c : chunks) {
            any_soft |= c.soft > 0 || c.msoft > 0;
            any_failed |= c.failed;
        }
        if (any_soft && !any_failed) {
            for (auto& c : chunks) {
                Chunk fresh;
                fresh.b = c.b;
                fresh.e = c.e;
                c = std::move(fresh);
            }
            parallel_for(threads, n_chunks, [&](int, int64_t cb, int64_t ce) {
                for (int64_t i = cb; i < ce; i++) parse_chunk(chunks[i], field, af_info, ns, true);
            });
        }
    }
    // counts and the first failure in file order
    uint64_t before = 0;
    for (auto& c : chunks) {
        if (c.failed) {
            std::string m = c.fail_kind;
            const size_t at = m.find("%R");
            if (at != std::string::npos) m.replace(at, 2, std::to_string(before + c.fail_rec));
            err = m;
            out.total = before + c.fail_rec;
            return 1;
        }
        before += c.total;
        out.total += c.total;
        out.not_snp += c.not_snp;
        out.multi += c.multi;
        out.soft += c.soft;
        out.incomplete += c.incomplete;
        out.n_sites += c.kept;
    }
    // sample-major codes of the biallelic and of the multi-allelic records
    const int64_t nv = out.n_sites;
    out.codes.allocate((size_t)(nv * (int64_t)ns));
    transpose_chunks(threads, ns, nv, out.codes.data(), chunks,
                     [](const Chunk& c) { return std::make_pair(c.rows.data(), c.kept); });
    bool any_soft = out.soft > 0;
    for (auto& c : chunks) any_soft |= c.msoft > 0;
    if (field != 'T' && any_soft) {
        // sample-major likelihoods [s][v][3], each thread a range of samples
        out.gl.resize((size_t)(nv * (int64_t)ns * 3));
        std::vector<int64_t> first((size_t)chunks.size() + 1, 0);
        for (size_t i = 0; i < chunks.size(); i++) first[i + 1] = first[i] + chunks[i].kept;
        parallel_for(threads, (int64_t)ns, [&](int, int64_t s0, int64_t s1) {
            for (size_t i = 0; i < chunks.size(); i++) {
                const double* lr = chunks[i].lrows.data();
                for (int64_t s = s0; s < s1; s++)
                    for (int64_t v = 0; v < chunks[i].kept; v++)
                        std::memcpy(out.gl.data() + ((size_t)s * nv + first[i] + v) * 3,
                                    lr + ((size_t)v * ns + s) * 3, sizeof(double) * 3);
            }
        });
    }
    out.n_multi = 0;
    for (auto& c : chunks) out.n_multi += c.mkept;
    out.mcodes.allocate((size_t)(out.n_multi * (int64_t)ns));
    transpose_chunks(threads, ns, out.n_multi, out.mcodes.data(), chunks,
                     [](const Chunk& c) { return std::make_pair(c.mrows.data(), c.mkept); });
    for (auto& c : chunks) {
        out.malleles.insert(out.malleles.end(), c.malleles.begin(), c.malleles.end());
        out.maf.insert(out.maf.end(), c.maf.begin(), c.maf.end());
        out.tri += c.tri;
        out.tetra += c.tetra;
        out.tri_full += c.tri_full;
        out.tetra_full += c.tetra_full;
        out.multi_incomplete += c.mincomplete;
        out.multi_dropped += c.multi_dropped;
        out.multi_soft += c.msoft;
    }
    if (field != 'T' && any_soft && out.n_multi > 0) {
        // sample-major likelihoods [s][record][10], each thread a range of samples
        const int64_t nm = out.n_multi;
        out.mgl.resize((size_t)(nm * (int64_t)ns * 10));
        std::vector<int64_t> first((size_t)chunks.size() + 1, 0);
        for (size_t i = 0; i < chunks.size(); i++) first[i + 1] = first[i] + chunks[i].mkept;
        parallel_for(threads, (int64_t)ns, [&](int, int64_t s0, int64_t s1) {
            for (size_t i = 0; i < chunks.size(); i++) {
                const double* lr = chunks[i].mlrows.data();
                for (int64_t s = s0; s < s1; s++)
                    for (int64_t v = 0; v < chunks[i].mkept; v++)
                        std::memcpy(out.mgl.data() + ((size_t)s * nm + first[i] + v) * 10,
                                    lr + ((size_t)v * ns + s) * 10, sizeof(double) * 10);
            }
        });
    }
    if (af_info) {
        out.af.reserve((size_t)(2 * nv));
        for (auto& c : chunks) out.af.insert(out.af.end(), c.af.begin(), c.af.end());
    }
    return 0;
}

void pack_2bit(const VcfData& d, int threads, uint32_t* codes2, uint32_t* observed) {
    const int64_t ns = (int64_t)d.samples.size(), nv = d.n_sites;
    const int64_t w2 = (nv + 15) / 16, wm = (nv + 31) / 32;
    parallel_for(host_threads(threads), ns, [&](int, int64_t s0, int64_t s1) {
        for (int64_t s = s0; s < s1; s++) {
            const uint8_t* row = d.codes.data() + s * nv;
            uint32_t* c2 = codes2 + s * w2;
            uint32_t* ob = observed + s * wm;
            for (int64_t w = 0; w < wm; w++) {
                uint32_t lo = 0, hi = 0, seen = 0;
                const int64_t v0 = w * 32;
                const int n = (int)std::min<int64_t>(32, nv - v0);
                for (int k = 0; k < n; k++) {
                    const uint32_t c = row[v0 + k];
                    const uint32_t called = c < 3 ? 1u : 0u;
                    const uint32_t cc = called ? c : 0u;
                    seen |= called << k;
                    if (k < 16) lo |= cc << (2 * k);
                    else hi |= cc << (2 * (k - 16));
                }
                ob[w] = seen;
                c2[2 * w] = lo;
                if (2 * w + 1 < w2) c2[2 * w + 1] = hi;
            }
        }
    });
}

}  // namespace kg

// ------------------------------------------------------------------- C ABI
struct kg_vcf {
    kg::VcfData d;
    std::string err;
};

extern "C" int kg_vcf_read(const char* path, const char* field, int af_info, int threads, kg_vcf** out) {
    if (!out) return KG_EINVAL;
    *out = nullptr;
    kg_vcf* v = new (std::nothrow) kg_vcf;
    if (!v) return KG_ENOMEM;
    *out = v;
    try {
        if (!path || !field) {
            v->err = "path and field are required";
            return KG_EINVAL;
        }
        const std::string f(field);
        char fc;
        if (f == "GT") fc = 'T';
        else if (f == "GL") fc = 'L';
        else if (f == "PL") fc = 'P';
        else {
            v->err = "field must be GT, GL or PL";
            return KG_EINVAL;
        }
        if (kg::read_vcf(path, fc, af_info != 0, threads, v->d, v->err)) return KG_EINVAL;
        return KG_OK;
    } catch (const std::bad_alloc&) {
        v->err = "out of host memory";
        return KG_ENOMEM;
    } catch (const std::exception& e) {
        v->err = e.what();
        return KG_EINVAL;
    }
}

extern "C" const char* kg_vcf_error(const kg_vcf* v) { return v ? v->err.c_str() : "null handle"; }

extern "C" int kg_vcf_info(const kg_vcf* v, int64_t* n_samples, int64_t* n_sites, uint64_t* counts) {
    if (!v) return KG_EINVAL;
    if (n_samples) *n_samples = (int64_t)v->d.samples.size();
    if (n_sites) *n_sites = v->d.n_sites;
    if (counts) {
        counts[0] = v->d.total;
        counts[1] = v->d.not_snp;
        counts[2] = v->d.multi;
        counts[3] = v->d.soft;
        counts[4] = v->d.incomplete;
        counts[5] = v->d.tri;
        counts[6] = v->d.tetra;
    }
    return KG_OK;
}

extern "C" int kg_vcf_codes(const kg_vcf* v, uint8_t* codes, double* af) {
    if (!v) return KG_EINVAL;
    if (codes && !v->d.codes.empty()) std::memcpy(codes, v->d.codes.data(), v->d.codes.size());
    if (af) {
        if (v->d.af.empty()) return KG_EINVAL;
        std::memcpy(af, v->d.af.data(), sizeof(double) * v->d.af.size());
    }
    return KG_OK;
}

extern "C" int kg_vcf_likelihoods(const kg_vcf* v, double* gl) {
    if (!v || !gl) return KG_EINVAL;
    if (v->d.gl.empty()) return KG_ENOTFOUND;
    std::memcpy(gl, v->d.gl.data(), sizeof(double) * v->d.gl.size());
    return KG_OK;
}

extern "C" int kg_vcf_codes_2bit(const kg_vcf* v, uint32_t* codes2, uint32_t* observed) {
    if (!v || !codes2 || !observed) return KG_EINVAL;
    kg::pack_2bit(v->d, 0, codes2, observed);
    return KG_OK;
}

extern "C" int kg_vcf_likelihoods_multiallelic(const kg_vcf* v, int n_alleles, double* gl) {
    if (!v || (n_alleles != 3 && n_alleles != 4)) return KG_EINVAL;
    if (v->d.mgl.empty()) return KG_ENOTFOUND;
    if (!gl) return KG_OK;
    const int ng = n_alleles * (n_alleles + 1) / 2;
    const int64_t ns = (int64_t)v->d.samples.size(), nm = v->d.n_multi;
    int64_t k = 0;
    std::vector<int64_t> sel;
    for (int64_t r = 0; r < nm; r++)
        if (v->d.malleles[(size_t)r] == n_alleles) sel.push_back(r);
    const int64_t nk = (int64_t)sel.size();
    for (int64_t s = 0; s < ns; s++)
        for (k = 0; k < nk; k++)
            std::memcpy(gl + (s * nk + k) * ng, v->d.mgl.data() + ((size_t)s * nm + sel[(size_t)k]) * 10,
                        sizeof(double) * ng);
    return KG_OK;
}

extern "C" int kg_vcf_multiallelic(const kg_vcf* v, uint8_t* gidx, uint8_t* n_alleles, double* af) {
    if (!v) return KG_EINVAL;
    if (gidx && !v->d.mcodes.empty()) std::memcpy(gidx, v->d.mcodes.data(), v->d.mcodes.size());
    if (n_alleles && !v->d.malleles.empty()) std::memcpy(n_alleles, v->d.malleles.data(), v->d.malleles.size());
    if (af) {
        if (v->d.maf.size() != 4 * (size_t)v->d.n_multi) return KG_EINVAL;
        if (!v->d.maf.empty()) std::memcpy(af, v->d.maf.data(), sizeof(double) * v->d.maf.size());
    }
    return KG_OK;
}

extern "C" const char* kg_vcf_sample(const kg_vcf* v, int64_t i) {
    if (!v || i < 0 || i >= (int64_t)v->d.samples.size()) return nullptr;
    return v->d.samples[(size_t)i].c_str();
}

extern "C" void kg_vcf_free(kg_vcf* v) { delete v; }
