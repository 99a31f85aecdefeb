// Minimizer-bucketed table (format MZ8): the key -> (bucket, slot) map.
//
// A canonical k-mer C is filed under its minimizer: among C's w = k - 15
// 16-mers, the one whose canonical form has the smallest bijective 32-bit
// hash h (ties: the leftmost in C). Consecutive reference positions mostly
// share their minimizer (runs of up to w positions), so their probes fall in
// one place of the table.
//
// The table is an array of 128-byte lines of four 32-byte sectors; a sector
// is a B8x32 bucket. The minimizer picks the line and C itself picks one of
// its four sectors, so a minimizer's k-mers (up to w of them, too many for
// one 8-slot sector) spread over the line, and a warp's loads for a run of
// positions touch one DRAM line.
//
// The slot value identifies C exactly inside its line: with g = spread(h)
// (a bijection of 32-bit values), line = floor(g * nLines / 2^32), so the
// low hbits of g single out g, hence h and the canonical minimizer M, among
// the line's interval; C is then M at offset o, in orientation s (M or its
// reverse complement), with the other k-16 bases around it:
//   slot = ((o << 1 | s) << 2(k-16) | C-without-the-16-mer) << hbits | (g mod 2^hbits)
// which must fit 31 bits (B8x32 sentinels): nLines >= 2^(2k-26).
#pragma once

#include "ibs_core.cuh"

namespace ibs {
namespace mz {

constexpr uint32_t M = 16; // minimizer length: a 16-mer is one 32-bit word

IBS_HD uint32_t w_of(uint32_t k) { return k - M + 1; }

IBS_HD uint32_t brev32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0f0f0f0fu) | ((x & 0x0f0f0f0fu) << 4);
    x = ((x >> 8) & 0x00ff00ffu) | ((x & 0x00ff00ffu) << 8);
    return (x >> 16) | (x << 16);
#endif
}

// Reverse complement of a 16-mer code (first base in the high bits).
IBS_HD uint32_t rc16(uint32_t v)
{
    uint32_t y = brev32(v);
    y = ((y >> 1) & 0x55555555u) | ((y & 0x55555555u) << 1);
    return ~y;
}

IBS_HD uint32_t canon16(uint32_t v)
{
    const uint32_t r = rc16(v);
    return v < r ? v : r;
}

IBS_HD uint32_t hash16(uint32_t canonical) { return (uint32_t)perm_hash(canonical, 32); }

// The 16-mer of C (2k-bit code, first base high) at offset o.
IBS_HD uint32_t mmer_at(uint64_t C, uint32_t k, uint32_t o)
{
    return (uint32_t)(C >> (2 * (k - M - o)));
}

// (o, s, C without the 16-mer) part of the slot value, given the offset.
IBS_HD uint32_t slot_high(uint64_t C, uint32_t k, uint32_t o)
{
    const uint32_t mm = mmer_at(C, k, o);
    const uint32_t s = mm != canon16(mm) ? 1u : 0u;
    const uint32_t rbits = 2 * (k - M - o);                    // bases right of the 16-mer
    const uint64_t right = rbits ? (C & ((1ull << rbits) - 1)) : 0;
    const uint64_t left = C >> (2 * (k - o));                  // bases left of it (2o bits)
    const uint64_t rest = (left << rbits) | right;             // 2(k-16) bits
    return (uint32_t)((((uint64_t)o << 1 | s) << (2 * (k - M))) | rest);
}

// Minimizer of C by brute force (table build, single probes): hash and
// leftmost offset.
IBS_HD void minimizer(uint64_t C, uint32_t k, uint32_t &h, uint32_t &o)
{
    h = 0xffffffffu;
    o = 0;
    bool first = true;
    for (uint32_t j = 0; j < w_of(k); ++j) {
        const uint32_t v = hash16(canon16(mmer_at(C, k, j)));
        if (first || v < h) {
            h = v;
            o = j;
            first = false;
        }
    }
}

// A minimizer's hash is the smallest of w hashes, so minimizer hashes crowd
// towards 0; the line is taken from a bijective remix of it, which is
// uniform over the minimizers again. Being a bijection, the remix (hence h)
// is still identified by (line, its low hbits).
IBS_HD uint32_t spread(uint32_t h) { return (uint32_t)perm_hash(h ^ 0x6a09e667u, 32); }

constexpr uint32_t kSectorsPerLine = 4;

IBS_HD uint64_t line_of_h(uint32_t h, uint64_t nLines) { return ((uint64_t)spread(h) * nLines) >> 32; }

// Sector of C inside its line: two well-mixed bits of the code.
IBS_HD uint32_t sector_of(uint64_t C) { return (uint32_t)((C * 0x9e3779b97f4a7c15ull) >> 62); }

// Bucket (32-byte sector index) of canonical k-mer C with minimizer hash h.
IBS_HD uint64_t bucket_of_h(uint32_t h, uint64_t C, uint64_t nBuckets)
{
    return line_of_h(h, nBuckets / kSectorsPerLine) * kSectorsPerLine + sector_of(C);
}

IBS_HD uint32_t slot_value(uint32_t high, uint32_t h, uint32_t hbits)
{
    return (high << hbits) | (spread(h) & (uint32_t)key_mask(hbits));
}

// Slot value and bucket of a canonical k-mer.
IBS_HD void locate(uint64_t C, const TableGeom &g, uint64_t &bucket, uint32_t &slot)
{
    uint32_t h, o;
    minimizer(C, g.k, h, o);
    bucket = bucket_of_h(h, C, g.nBuckets);
    slot = slot_value(slot_high(C, g.k, o), h, g.fpBits);
}

} // namespace mz
} // namespace ibs
