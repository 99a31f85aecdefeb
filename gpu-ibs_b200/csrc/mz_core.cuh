// Minimizer-bucketed table (format MZ8): the key -> (bucket, slot) map.
//
// A canonical k-mer C is filed under its minimizer: among C's w = k - m + 1
// m-mers (m = k - 6 from k = 22, else 16), the one whose canonical form has
// the smallest rank key (29 bits derived from the m-mer's line hash, below),
// ties going to the leftmost in C. Consecutive
// reference positions mostly share their minimizer (runs of up to w
// positions), so their probes fall in one place of the table. m grows with k so that a minimizer rarely occurs at
// two loci of a large genome (4^19 19-mers against 2e9 positions), which
// would pile two runs into one place.
//
// The table is an array of 128-byte lines of four 32-byte sectors; a sector
// is a B8x32 bucket (format MZ8) or a B6x40 bucket (format MZ6). The
// minimizer picks the line and C itself picks one of its four sectors, so a
// minimizer's k-mers spread over the line and a warp's loads for a run of
// positions touch one DRAM line.
//
// The slot value identifies C exactly inside its line: with g = line_hash(M)
// (a bijection of the 2m-bit canonical minimizer M), line = the top 32 bits
// of g scaled to [0, nLines), so the low hbits = 2m - floor(log2(nLines))
// bits of g single out g, hence M, among the line's interval; C is then M at
// offset o (< w <= 8), in orientation s (M or its reverse complement), with
// the other k - m bases around it:
//   slot = ((o << 1 | s) << 2(k-m) | C-without-the-m-mer) << hbits | (g mod 2^hbits)
// which has 2k + 4 - floor(log2(nLines)) bits and must fit the sector's slots: 31
// bits in B8x32 sectors (format MZ8, the sentinels above), nLines >=
// 2^(2k-27); 40 bits in B6x40 sectors (format MZ6, for k up to 31), nLines
// >= 2^(2k-36).
#pragma once

#include "ibs_core.cuh"

namespace ibs {
namespace mz {

constexpr uint32_t kSectorsPerLine = 4;

IBS_HD uint32_t m_of(uint32_t k) { return k >= 22 ? k - 6 : 16; }
IBS_HD uint32_t w_of(uint32_t k) { return k - m_of(k) + 1; }

IBS_HD uint64_t brev64(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return __brevll(x);
#else
    x = ((x >> 1) & 0x5555555555555555ull) | ((x & 0x5555555555555555ull) << 1);
    x = ((x >> 2) & 0x3333333333333333ull) | ((x & 0x3333333333333333ull) << 2);
    x = ((x >> 4) & 0x0f0f0f0f0f0f0f0full) | ((x & 0x0f0f0f0f0f0f0f0full) << 4);
    x = ((x >> 8) & 0x00ff00ff00ff00ffull) | ((x & 0x00ff00ff00ff00ffull) << 8);
    x = ((x >> 16) & 0x0000ffff0000ffffull) | ((x & 0x0000ffff0000ffffull) << 16);
    return (x >> 32) | (x << 32);
#endif
}

// Reverse complement of an m-mer code (first base in the high bits).
IBS_HD uint64_t rc_m(uint64_t v, uint32_t m)
{
    uint64_t y = brev64(v);
    y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
    return ~y >> (64 - 2 * m);
}

IBS_HD uint64_t canon_m(uint64_t v, uint32_t m)
{
    const uint64_t r = rc_m(v, m);
    return v < r ? v : r;
}

// The line hash of a canonical m-mer: a bijection of the 2m-bit values, two
// multiply-xorshift rounds, so the lines stay uniform over the minimizers.
IBS_HD uint64_t line_hash(uint64_t canonical, uint32_t m)
{
    const uint64_t mask = key_mask(2 * m);
    uint64_t x = (canonical * 0xd6e8feb86659fd93ull) & mask;
    x ^= x >> m;
    x = (x * 0xbf58476d1ce4e5b9ull) & mask;
    x ^= x >> m;
    return x;
}

// The key minimizers are chosen by: an odd 32-bit multiple of the line
// hash's low 32 bits, with its low 3 bits cleared. Cheap on purpose: the scan
// computes one per reference position, and it packs a window offset into the
// 3 free bits so that one integer minimum per offset finds the leftmost (or,
// on the other strand, the rightmost) smallest key. The line index comes
// from the line hash's high bits; for every fixed line the multiples of its
// low bits are spread evenly over the key range (a golden-ratio multiplier),
// so picking small keys does not crowd lines.
IBS_HD uint32_t rank_key_of(uint64_t lineHash) { return ((uint32_t)lineHash * 0x9e3779b1u) & ~7u; }

IBS_HD uint32_t rank_key(uint64_t canonical, uint32_t m) { return rank_key_of(line_hash(canonical, m)); }

// The m-mer of C (2k-bit code, first base high) at offset o.
IBS_HD uint64_t mmer_at(uint64_t C, uint32_t k, uint32_t o, uint32_t m)
{
    return (C >> (2 * (k - m - o))) & key_mask(2 * m);
}

// (o, s, C without the m-mer) part of the slot value: the minimizer's
// offset o in C and its orientation s there (1 when it reads as the reverse
// complement of its canonical form), then the k - m other bases: C rotated
// left by 2o bits inside its 2k puts the m-mer on top and below it the bases
// right of the m-mer followed by the o bases left of it. 2(k - m) + 4 <= 16
// bits; m >= 16 and o <= k - m keep both shifts below 32.
IBS_HD uint32_t slot_high(uint64_t C, uint32_t k, uint32_t o, uint32_t s)
{
    const uint32_t m = m_of(k);
    const uint32_t lo = (uint32_t)C, hi = (uint32_t)(C >> 32);
    const uint32_t rest = ((lo << (2 * o)) | (hi >> (2 * k - 32 - 2 * o))) & (uint32_t)key_mask(2 * (k - m));
    return (((o << 1) | s) << (2 * (k - m))) | rest;
}

// Minimizer offset of C by brute force (table build, single probes): the
// leftmost m-mer with the smallest rank key.
IBS_HD uint32_t minimizer_offset(uint64_t C, uint32_t k)
{
    const uint32_t m = m_of(k);
    uint32_t best = 0xffffffffu, o = 0;
    for (uint32_t j = 0; j < w_of(k); ++j) {
        const uint32_t v = rank_key(canon_m(mmer_at(C, k, j, m), m), m);
        if (j == 0 || v < best) {
            best = v;
            o = j;
        }
    }
    return o;
}

// Sector of C inside its line: the top two bits of a golden-ratio multiple
// of the code's two halves folded together.
IBS_HD uint32_t sector_of(uint64_t C) { return (((uint32_t)C ^ (uint32_t)(C >> 32)) * 0x9e3779b1u) >> 30; }

// Line of a minimizer with line hash g (2m >= 32 bits) among nLines < 2^32:
// the top 32 bits of g scaled to [0, nLines). Those of one line form an
// interval of at most ceil(2^32 / nLines) values, so the g of a line form an
// interval of at most 2^(2m - floor(log2 nLines)) = 2^hbits values and
// g mod 2^hbits singles g out in its line.
IBS_HD uint64_t line_of(uint64_t g, uint32_t m, uint64_t nLines)
{
    const uint32_t top = (uint32_t)(g >> (2 * m - 32));
#if defined(__CUDA_ARCH__)
    return __umulhi(top, (uint32_t)nLines);
#else
    return ((uint64_t)top * (uint32_t)nLines) >> 32;
#endif
}

// Bucket (32-byte sector index) and slot value of canonical k-mer C whose
// minimizer sits at offset o with orientation s and line hash g.
// hbits = 2m - floor(log2(nLines)).
IBS_HD void place(uint64_t C, uint32_t k, uint32_t o, uint32_t s, uint64_t g, uint64_t nBuckets,
                  uint32_t hbits, uint64_t &bucket, uint64_t &slot)
{
    bucket = line_of(g, m_of(k), nBuckets / kSectorsPerLine) * kSectorsPerLine + sector_of(C);
    slot = ((uint64_t)slot_high(C, k, o, s) << hbits) | (g & key_mask(hbits));
}

// The same as place() where the slot value fits 32 bits (MZ8 sectors, joint
// minimizer lines: hbits < 32 and the slot below 2^32 by their line counts),
// in 32-bit arithmetic. Only bits 0 .. 2m-1 of g are read, so flag bits above
// them do not matter.
IBS_HD void place32(uint64_t C, uint32_t k, uint32_t o, uint32_t s, uint64_t g, uint64_t nBuckets,
                    uint32_t hbits, uint64_t &bucket, uint64_t &slot)
{
    bucket = line_of(g, m_of(k), nBuckets / kSectorsPerLine) * kSectorsPerLine + sector_of(C);
    const uint32_t low = (uint32_t)g & ((1u << hbits) - 1u);
    slot = (slot_high(C, k, o, s) << hbits) | low;
}

// Slot value and bucket of a canonical k-mer (the build side, and single
// probes): everything from C itself.
IBS_HD void locate(uint64_t C, const TableGeom &g, uint64_t &bucket, uint64_t &slot)
{
    const uint32_t m = m_of(g.k);
    const uint32_t o = minimizer_offset(C, g.k);
    const uint64_t mm = mmer_at(C, g.k, o, m);
    const uint64_t cm = canon_m(mm, m);
    place(C, g.k, o, mm != cm ? 1u : 0u, line_hash(cm, m), g.nBuckets, g.fpBits, bucket, slot);
}

} // namespace mz
} // namespace ibs
