// kg_vcf.h — multithreaded VCF reader for the CLI and the C ABI.
//
// Reads biallelic SNP records of a VCF 4.x file (plain, gzip or bgzip) into
// per-sample genotype codes (0 = 0/0, 1 = 0/1, 2 = 1/1, 3 = missing), with the
// reference's record rules (src/vcf.rs:96-236): records whose REF or ALT is not
// a single base are skipped; tri- and tetra-allelic records are kept apart as
// genotype indices in the VCF order (the reference's gt3 / gt4 and gl3 / gl4),
// 255 for a missing call; GT calls are diploid allele indices separated by '/'
// or '|' ('.' = missing); GL/PL calls are likelihoods reduced to the most
// likely genotype (a row that is not one-hot to 25.5 log10 units is counted as
// soft).  BGZF blocks are
// inflated in parallel; the text is cut at line boundaries and the chunks are
// parsed in parallel, then merged in file order.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace kg {

// A byte array that is not zero-filled on allocation (its writers touch every
// byte, from several threads).
class Bytes {
public:
    void allocate(size_t n) {
        p_.reset(new uint8_t[n ? n : 1]);
        n_ = n;
    }
    uint8_t* data() { return p_.get(); }
    const uint8_t* data() const { return p_.get(); }
    size_t size() const { return n_; }
    bool empty() const { return n_ == 0; }

private:
    std::unique_ptr<uint8_t[]> p_;
    size_t n_ = 0;
};

struct VcfData {
    std::vector<std::string> samples;
    int64_t n_sites = 0;            // kept (biallelic SNP) records
    Bytes codes;                    // sample-major: codes[s * n_sites + v]
    std::vector<double> af;         // with allele frequencies from INFO/AF: [REF, ALT] per kept site
    uint64_t total = 0, not_snp = 0, multi = 0, soft = 0;
    uint64_t incomplete = 0;        // SNP records with at least one missing call
    // tri- and tetra-allelic records
    int64_t n_multi = 0;
    Bytes mcodes;                   // sample-major genotype indices (VCF order, 255 = missing), mcodes[s * n_multi + v]
    std::vector<uint8_t> malleles;  // allele count per record (3 or 4)
    std::vector<double> maf;        // with INFO/AF: 4 per record, [REF, ALT1, ALT2, ALT3 or 0]
    uint64_t tri = 0, tetra = 0;    // kept records by allele count
    uint64_t tri_full = 0, tetra_full = 0;   // of those, the ones every sample calls
    uint64_t multi_incomplete = 0;  // kept records with a missing call
    uint64_t multi_dropped = 0;     // GT records dropped: a malformed call after a missing one
    uint64_t multi_soft = 0;        // GL/PL likelihood rows of these records that are not one-hot
    // GL/PL with a soft row: their linear-scale likelihoods, [s][record][10]
    // (G used, NaN after and where missing); empty otherwise
    std::vector<double> mgl;
    // GL/PL with a soft row: the linear-scale likelihoods, sample-major
    // gl[(s * n_sites + v) * 3 + g] (NaN where missing); empty otherwise
    std::vector<double> gl;
};

// The codes in the packed form kg_load_genotypes_2bit takes: per sample
// ceil(n_sites / 16) words of 2-bit codes (site s at bits 2 (s % 16) of word
// s / 16, 0 where missing) and ceil(n_sites / 32) words of the observed mask
// (bit s % 32 of word s / 32).  Samples in parallel over `threads`.
void pack_2bit(const VcfData& d, int threads, uint32_t* codes2, uint32_t* observed);

// field: 'T' GT, 'L' GL, 'P' PL.  af_info: read INFO/AF (an error when absent).
// threads <= 0: all hardware threads.  Returns 0, or 1 with err set (the
// message of the first bad record in file order).
int read_vcf(const std::string& path, char field, bool af_info, int threads, VcfData& out, std::string& err);

}  // namespace kg
