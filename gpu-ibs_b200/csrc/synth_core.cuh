// Counter-based synthetic inputs: every base, N run, SNP and extra k-mer is a
// pure function of (seed, stream, index), so the CPU and GPU generators give
// identical data and any slice can be generated independently.
//
// Reference: contig c, base i = 2-bit field (i % 32) of rnd(seed, S_BASE+c,
// i/32); N runs at rnd-drawn starts and lengths; lowercase runs (FASTA text
// only). Sample: a copy of the reference cut into blocks whose SNP rate is
// drawn per block from up to four classes; a block is present with
// probability present_frac; introgression blocks override the rate; a
// SNP replaces the base by one of the three others. The sample's k-mer set
// is the canonical k-mers of the copy at positions whose k reference bases
// are ACGT and whose block is present, plus random canonical k-mers.
#pragma once

#include <cstdint>

#include "ibs_core.cuh"

namespace ibs {
namespace synth {

enum : uint64_t {
    S_BASE = 0x1000,
    S_NRUN = 0x100000,
    S_LOWER = 0x200000,
    S_BLOCK = 0x300000,
    S_SNP = 0x400000,
    S_SNPB = 0x500000,
    S_PRESENT = 0x600000,
    S_RAND = 0x700000,
    S_COUNT = 0x800000,
};

IBS_HD uint64_t rnd(uint64_t seed, uint64_t stream, uint64_t i)
{
    return fmix64(fmix64(seed ^ (stream * 0x9e3779b97f4a7c15ull)) + i * 0xd1b54a32d192ed03ull);
}

// Base word w (bases 32w..32w+31) of contig c before N masking.
IBS_HD uint64_t base_word(uint64_t seed, uint32_t c, uint64_t w) { return rnd(seed, S_BASE + c, w); }

struct SampleParams {
    uint64_t seed;
    uint32_t k;
    uint32_t nClasses;
    uint64_t blockLen;
    uint64_t classCut[4];  // cumulative class probabilities scaled to 2^64 (last = ~0)
    uint64_t classThr[4];  // SNP probability per base scaled to 2^64
    uint64_t presentThr;   // block present if rnd < presentThr (~0 = always)
    uint64_t introThr;     // SNP threshold inside introgression blocks
};

IBS_HD uint64_t snp_threshold_of_block(const SampleParams &s, uint32_t c, uint64_t blk)
{
    const uint64_t u = rnd(s.seed, S_BLOCK + c, blk);
    for (uint32_t j = 0; j + 1 < s.nClasses; ++j)
        if (u < s.classCut[j])
            return s.classThr[j];
    return s.classThr[s.nClasses - 1];
}

IBS_HD bool block_present(const SampleParams &s, uint32_t c, uint64_t blk)
{
    return s.presentThr == ~0ull || rnd(s.seed, S_PRESENT + c, blk) < s.presentThr;
}

// The sample's base at contig position i given the reference base and the
// SNP threshold of its block.
IBS_HD uint32_t copy_base(const SampleParams &s, uint32_t c, uint64_t i, uint32_t refBase,
                          uint64_t thr)
{
    if (thr && rnd(s.seed, S_SNP + c, i) < thr)
        return (refBase + 1 + (uint32_t)(rnd(s.seed, S_SNPB + c, i) % 3)) & 3;
    return refBase;
}

IBS_HD uint64_t canonical_of(uint64_t code, uint32_t k)
{
    // reverse complement of a 2k-bit code
    uint64_t rc = 0, x = code;
    for (uint32_t t = 0; t < k; ++t) {
        rc = (rc << 2) | (3 - (x & 3));
        x >>= 2;
    }
    return code < rc ? code : rc;
}

// KMC counter of a k-mer: uniform 2..255.
IBS_HD uint32_t count_of(uint64_t seed, uint64_t code) { return 2 + (uint32_t)(rnd(seed, S_COUNT, code) % 254); }

// ---- KMC minimizer signature (the norm table of KMC's CMmer: an m-mer is
// "allowed" unless it ends in TTT, TGT or TG*, contains AA after its first
// symbol, or starts with AAA, ACA or *AA; norm[m] = min(m, rc(m)) over the
// allowed ones, 4^len when neither is) ---------------------------------------
IBS_HD bool mmer_allowed(uint32_t m, uint32_t len)
{
    if ((m & 0x3f) == 0x3f || (m & 0x3f) == 0x3b || (m & 0x3c) == 0x3c)
        return false;
    for (uint32_t j = 0; j < len - 3; ++j) {
        if ((m & 0xf) == 0)
            return false;
        m >>= 2;
    }
    if (m == 0 || m == 0x04 || (m & 0xf) == 0)
        return false;
    return true;
}

IBS_HD uint32_t norm_value(uint32_t m, uint32_t len)
{
    const uint32_t special = 1u << (2 * len);
    uint32_t rev = 0, x = m;
    for (uint32_t j = 0; j < len; ++j) {
        rev = (rev << 2) | (3 - (x & 3));
        x >>= 2;
    }
    const uint32_t a = mmer_allowed(m, len) ? m : special;
    const uint32_t b = mmer_allowed(rev, len) ? rev : special;
    return a < b ? a : b;
}

IBS_HD uint32_t signature_of(uint64_t code, uint32_t k, uint32_t sigLen, const uint32_t *norm)
{
    const uint32_t mmask = (1u << (2 * sigLen)) - 1;
    uint32_t str = 0, best = 0xffffffffu;
    for (uint32_t i = 0; i < k; ++i) {
        str = ((str << 2) | (uint32_t)((code >> (2 * (k - 1 - i))) & 3)) & mmask;
        if (i + 1 >= sigLen) {
            const uint32_t v = norm[str];
            best = v < best ? v : best;
        }
    }
    return best;
}

// Signature -> bin map written into the .kmc_pre signature map.
IBS_HD uint32_t bin_of_signature(uint32_t sig, uint32_t nBins) { return sig % nBins; }

} // namespace synth
} // namespace ibs
