// Wide-key tables and codes: k-mers of 33 <= k <= 64 bases.
//
// The reference takes such k through its string path (k > 32 routes every
// database to getStatsFromSequenceLegacy, src/KmerDatabase.hpp:100-124 and
// :675-708): canonical k-mers as strings, each looked up in the KMC
// database. Here the canonical k-mer is a 2k-bit code held in two 64-bit
// words (lo = bits 0..63, hi = the rest; first base most significant, so
// the integer order is the string order of ACGT), and the table holds whole
// keys: no quotienting, since a 128-bit key space has no cheap bijection
// whose remainder fits a slot.
//
// Layout (format FMT_WIDE): 128-byte lines of eight 16-byte slots
// {lo, hi}; an empty slot is all ones in both words (never a canonical
// code: all ones is the all-T k-mer, whose reverse complement all-A is
// smaller; the build leaves out a key equal to it, which no scan asks for).
// The lines form up to kMaxLevels levels, each with its own line hash: level
// 0 holds the keys at about 4 per line; the keys of lines that got more than
// 8 go to level 1, sized at about 2 per line, and so on until none is left.
// A probe reads its level-0 line; a hit or an empty slot ends it, a full
// line sends it on to the next level.
#pragma once

#include <cuda_runtime.h>

#include "ibs_core.cuh"

namespace ibs {
namespace wide {

constexpr uint32_t kSlots = 8;
constexpr uint32_t kMaxLevels = 12;
constexpr uint64_t kEmpty = ~0ull;

// A table's levels: each its own device array of lines[L] lines of kSlots
// {lo, hi} slots.
struct View {
    uint32_t k, nLevels;
    uint64_t lines[kMaxLevels];
    const ulonglong2 *slots[kMaxLevels];
};

// Line of a key in one level: a 64-bit mix of both words, scaled to the
// level's line count.
IBS_HD uint64_t line_of(uint64_t lo, uint64_t hi, uint32_t level, uint64_t nLines)
{
    const uint64_t h = fmix64(lo ^ fmix64(hi + 0x9e3779b97f4a7c15ull * (level + 1)));
    return mulhi64(h, nLines);
}

// 2-bit symbols of x in reverse order.
IBS_HD uint64_t rev2(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    uint64_t y = __brevll(x);
#else
    uint64_t y = x;
    y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
    y = ((y >> 2) & 0x3333333333333333ull) | ((y & 0x3333333333333333ull) << 2);
    y = ((y >> 4) & 0x0f0f0f0f0f0f0f0full) | ((y & 0x0f0f0f0f0f0f0f0full) << 4);
    y = ((y >> 8) & 0x00ff00ff00ff00ffull) | ((y & 0x00ff00ff00ff00ffull) << 8);
    y = ((y >> 16) & 0x0000ffff0000ffffull) | ((y & 0x0000ffff0000ffffull) << 16);
    y = (y >> 32) | (y << 32);
#endif
    return ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
}

// Canonical code of the 2k-bit little-endian base stream (xlo, xhi) (base 0
// in bits 0-1 of xlo; bits of xhi above 2k - 64 are ignored): the forward
// code is the stream with its symbols reversed, the reverse complement is
// the complemented stream; the smaller one, compared as 128-bit integers.
IBS_HD void canonical_of_stream(uint64_t xlo, uint64_t xhi, uint32_t k, uint64_t &clo, uint64_t &chi)
{
    const uint32_t d = 128 - 2 * k; // 0 <= d < 64
    const uint64_t ylo = rev2(xhi), yhi = rev2(xlo);
    const uint64_t fhi = yhi >> d;
    const uint64_t flo = d ? ((ylo >> d) | (yhi << (64 - d))) : ylo;
    const uint64_t rlo = ~xlo, rhi = ~xhi & key_mask(2 * k - 64);
    const bool fwd = fhi < rhi || (fhi == rhi && flo <= rlo);
    clo = fwd ? flo : rlo;
    chi = fwd ? fhi : rhi;
}

// Canonical code of the k-mer whose first base is packed base G, and
// whether its k bases are all ACGT, from the sequence words G / 32 .. + 2
// (w0..w2: the k-mer spans at most three) and the mask words G / 64 .. + 1.
IBS_HD void canonical_from_words(uint64_t w0, uint64_t w1, uint64_t w2, uint64_t m0, uint64_t m1, uint64_t G,
                                 uint32_t k, bool &acgt, uint64_t &clo, uint64_t &chi)
{
    const uint32_t sh = (uint32_t)(G & 31) * 2;
    const uint64_t xlo = (w0 >> sh) | ((w1 << (63 - sh)) << 1);
    const uint64_t xhi = (w1 >> sh) | ((w2 << (63 - sh)) << 1);
    const uint32_t ms = (uint32_t)(G & 63);
    const uint64_t mm = (m0 >> ms) | ((m1 << (63 - ms)) << 1);
    acgt = (mm & key_mask(k)) == 0;
    canonical_of_stream(xlo, xhi, k, clo, chi);
}

#if defined(__CUDACC__)
// The same reading the packed reference (the packed layout's tail padding
// covers the word after a contig's last).
__device__ __forceinline__ void canonical_at(const uint64_t *__restrict__ seq, const uint64_t *__restrict__ mask,
                                             uint64_t G, uint32_t k, bool &acgt, uint64_t &clo, uint64_t &chi)
{
    const uint64_t wi = G >> 5, mi = G >> 6;
    canonical_from_words(__ldg(seq + wi), __ldg(seq + wi + 1), __ldg(seq + wi + 2), __ldg(mask + mi),
                         __ldg(mask + mi + 1), G, k, acgt, clo, chi);
}

// Membership of one wide key, from level L0 on.
__device__ __forceinline__ bool lookup(const View &t, uint64_t lo, uint64_t hi, uint32_t L0 = 0)
{
    for (uint32_t L = L0; L < t.nLevels; ++L) {
        const ulonglong2 *p = t.slots[L] + line_of(lo, hi, L, t.lines[L]) * kSlots;
        bool hit = false, room = false;
#pragma unroll
        for (uint32_t s = 0; s < kSlots; ++s) {
            const ulonglong2 v = __ldg(p + s);
            hit |= (v.x == lo) & (v.y == hi);
            room |= (v.x == kEmpty) & (v.y == kEmpty);
        }
        if (hit)
            return true;
        if (room)
            return false;
    }
    return false;
}

// Membership of the warp's 32 keys (one per lane; lanes with want == false
// take part and get false). Level 0 is read cooperatively: in each of 8
// steps, the four 8-lane groups read four keys' lines, lane i of a group
// slot i, so one 16-byte load per lane covers four whole 128-byte lines
// (instead of 32 lines touched per load when every lane reads its own
// line); each group's 8-bit ballot slices say hit and empty slot to the key's
// lane. A key whose level-0 line is full without it goes on to level 1 alone.
// Every lane of the warp must call it.
__device__ __forceinline__ bool lookup_warp(const View &t, uint64_t lo, uint64_t hi, bool want, uint32_t lane)
{
    const uint64_t line = want ? line_of(lo, hi, 0, t.lines[0]) : 0; // line 0 exists in every table
    const ulonglong2 *base = t.slots[0] + (lane & 7);
    const uint32_t group = lane >> 3;
    uint32_t hitBits = 0, roomBits = 0;
#pragma unroll
    for (uint32_t g = 0; g < 8; ++g) {
        const uint32_t owner = 4 * g + group; // the key this lane's group reads in step g
        const uint64_t l = __shfl_sync(0xffffffffu, line, owner);
        const uint64_t klo = __shfl_sync(0xffffffffu, lo, owner);
        const uint64_t khi = __shfl_sync(0xffffffffu, hi, owner);
        const ulonglong2 v = __ldg(base + l * kSlots);
        const uint32_t m = __ballot_sync(0xffffffffu, (v.x == klo) & (v.y == khi));
        const uint32_t e = __ballot_sync(0xffffffffu, (v.x == kEmpty) & (v.y == kEmpty));
        if ((lane >> 2) == g) { // this lane's key is 4 g + (lane & 3), read by group lane & 3
            hitBits = (m >> (8 * (lane & 3))) & 0xffu;
            roomBits = (e >> (8 * (lane & 3))) & 0xffu;
        }
    }
    if (!want)
        return false;
    if (hitBits)
        return true;
    if (roomBits)
        return false;
    return lookup(t, lo, hi, 1);
}
#endif

} // namespace wide
} // namespace ibs
