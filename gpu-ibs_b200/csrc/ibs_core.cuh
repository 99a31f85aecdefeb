// Core definitions shared by the host and the device code of the B200 fastibs
// window scan: the bijective k-mer hash, the sector-sized bucket formats of
// the device table, and the window-statistics monoid.
//
// Statistics semantics follow the reference exactly: a window's positions
// are visited in order, invalid positions (a non-ACGT base in the k-mer) are
// skipped, a miss extends the current gap, a hit closes it
// (KmerDatabase::getStatsFromSequence, src/KmerDatabase.hpp:628-646;
// BitStats::run, src/gpu/EncodeProbeCore.hpp:338-370), and a closed gap of
// g misses adds Window::addVariationOriginal(g, k) (src/Window.hpp:29-36).
// Here that loop is restated as an associative fold so any partition of a
// window's positions (warps, spans, launches) gives the same row.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define IBS_HD __host__ __device__ __forceinline__
#else
#define IBS_HD inline
#endif

namespace ibs {

// ---------------------------------------------------------------------------
// Bijective hash of a 2k-bit canonical code onto [0, 2^(2k)).
// xorshift-right and multiplication by an odd constant are both bijections
// modulo 2^bits, so the composition is a permutation of the key space: the
// table can store only the low bits of the hash (the quotient rest) and still
// identify a key exactly.
// ---------------------------------------------------------------------------
IBS_HD uint64_t key_mask(uint32_t bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

IBS_HD uint64_t perm_hash(uint64_t x, uint32_t bits)
{
    const uint64_t m = key_mask(bits);
    const uint32_t s = (bits + 1) >> 1;
    x ^= x >> s;
    x = (x * 0xff51afd7ed558ccdull) & m;
    x ^= x >> s;
    x = (x * 0xc4ceb9fe1a85ec53ull) & m;
    x ^= x >> s;
    return x;
}

// 64-bit finalizer (the stash slot index; not required to be a bijection).
IBS_HD uint64_t fmix64(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

IBS_HD uint64_t mulhi64(uint64_t a, uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// ---------------------------------------------------------------------------
// Device table geometry. Bucket r holds keys whose hash h satisfies
// floor(h * nBuckets / 2^bits) == r: a contiguous hash interval of length
// <= ceil(2^bits / nBuckets) <= 2^fpBits, so the low fpBits bits of h are
// distinct inside a bucket and (bucket, h mod 2^fpBits) determines the key.
//
// Format B8x32 (fpBits <= 31): one 32-byte sector = 8 x u32 fingerprints.
//   EMPTY = 0xffffffff; slot 7 == OVERFLOW marks a bucket with more than 8
//   keys: it keeps 7 and the rest live in the stash.
// Format B6x40 (fpBits <= 40): one 32-byte sector = 6 x u32 fingerprint
//   high parts, 6 x u8 low parts, u8 count, u8 flags (bit0 = overflow).
// Stash: open addressing over whole codes, 4 x u64 per 32-byte bucket,
//   linear probing over buckets, EMPTY = ~0 (never a canonical code: the
//   all-T k-mer's reverse complement, all-A, is smaller).
// ---------------------------------------------------------------------------
enum : uint32_t {
    FMT_B8X32 = 1, FMT_B6X40 = 2, FMT_PANEL = 3, FMT_MZ8 = 4, FMT_AUTO_HASH = 5, FMT_MZ6 = 6,
    FMT_PANEL_MZ = 7, // joint table: P5x48 sectors on minimizer lines (panel_core.cuh)
    FMT_WIDE = 8      // 33 <= k <= 64: whole 128-bit keys on 128-byte lines (wide_core.cuh)
};
// Minimizer-line tables: B8x32 sectors (31-bit slot values) or B6x40 sectors
// (40-bit slot values, for larger k).
IBS_HD bool is_mz(uint32_t fmt) { return fmt == FMT_MZ8 || fmt == FMT_MZ6; }
constexpr uint32_t B8_EMPTY = 0xffffffffu;
constexpr uint32_t B8_OVERFLOW = 0xfffffffeu;
// Minimizer lines of B8x32 sectors (MZ8) keep a full sector's extra keys in
// its partner sector of the same line (index ^ 1) while that has free slots:
// slot 7 = B8_OVERFLOW says the extras are all there, B8_OVERFLOW_STASH that
// some went on to the stash. (A slot value identifies its k-mer inside the
// whole line, so the two sectors' keys never collide.)
constexpr uint32_t B8_OVERFLOW_STASH = 0xfffffffdu;
constexpr uint64_t STASH_EMPTY = ~0ull;

struct TableGeom {
    uint32_t k;        // k-mer length (<= 32; <= 64 for FMT_WIDE)
    uint32_t bits;     // 2k
    uint32_t fpBits;   // stored fingerprint width
    uint32_t format;   // FMT_*
    uint64_t nBuckets; // sector buckets
    uint64_t stashBuckets; // power of two, 0 when there is no stash
};

IBS_HD uint64_t bucket_of(uint64_t h, const TableGeom &g)
{
    return mulhi64(h << (64 - g.bits), g.nBuckets);
}

IBS_HD uint64_t fp_of(uint64_t h, const TableGeom &g) { return h & key_mask(g.fpBits); }

IBS_HD uint64_t stash_home(uint64_t code, uint64_t stashBuckets)
{
    return fmix64(code ^ 0x9e3779b97f4a7c15ull) & (stashBuckets - 1);
}

// ---------------------------------------------------------------------------
// Window statistics as a monoid. A segment of a window's positions is
// summarised by: valid positions, hits, misses before its first hit (lead),
// misses after its last hit (trail), and the count and distance sum of the
// gaps closed strictly inside it. Without a hit, lead == trail == total.
// ---------------------------------------------------------------------------
struct SegStats {
    uint32_t total, obs, lead, trail, gaps, pad;
    int64_t dist;
};

// Distance contributed by one closed gap of g misses
// (Window::addVariationOriginal, src/Window.hpp:29-36).
IBS_HD int64_t gap_distance(int64_t g, int k)
{
    int64_t d = g - (k - 1);
    if (d <= 0)
        d = d + 1 < 0 ? -(d + 1) : d + 1;
    return d;
}

IBS_HD SegStats seg_empty()
{
    SegStats s;
    s.total = s.obs = s.lead = s.trail = s.gaps = s.pad = 0;
    s.dist = 0;
    return s;
}

// a followed by b.
IBS_HD SegStats seg_combine(const SegStats &a, const SegStats &b, int k)
{
    SegStats r;
    r.total = a.total + b.total;
    r.obs = a.obs + b.obs;
    r.pad = 0;
    if (a.obs == 0 && b.obs == 0) {
        r.lead = r.trail = a.lead + b.lead;
        r.gaps = 0;
        r.dist = 0;
    } else if (a.obs == 0) {
        r.lead = a.lead + b.lead;
        r.trail = b.trail;
        r.gaps = b.gaps;
        r.dist = b.dist;
    } else if (b.obs == 0) {
        r.lead = a.lead;
        r.trail = a.trail + b.lead;
        r.gaps = a.gaps;
        r.dist = a.dist;
    } else {
        const uint32_t g = a.trail + b.lead;
        r.lead = a.lead;
        r.trail = b.trail;
        r.gaps = a.gaps + b.gaps + (g > 0 ? 1u : 0u);
        r.dist = a.dist + b.dist + (g > 0 ? gap_distance(g, k) : 0);
    }
    return r;
}

// Final row values of a whole window: the leading gap closes at the first
// hit, the trailing one at the window's end; without any hit the window is
// one gap of `total` misses.
struct WindowRow {
    int32_t start, end, total_kmers, observed_kmers, variations, kmer_distance;
};

// Statistics of up to 32 consecutive positions in 32-bit fields (a block of
// the scan, or a run of blocks whose counts stay below 2^32): the SegStats
// monoid without the 64-bit distance.
struct Seg32 {
    uint32_t total, obs, lead, trail, gaps, dist;
};

IBS_HD uint32_t popc32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return __popc(x);
#else
    return (uint32_t)__builtin_popcount(x);
#endif
}

// Index of the lowest set bit of x != 0.
IBS_HD uint32_t ctz32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return __ffs(x) - 1;
#else
    return (uint32_t)__builtin_ctz(x);
#endif
}

IBS_HD uint32_t clz32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return __clz(x);
#else
    return (uint32_t)__builtin_clz(x);
#endif
}

IBS_HD uint32_t gap_distance32(uint32_t g, int k)
{
    const int d = (int)g - (k - 1);
    return (uint32_t)(d > 0 ? d : (d + 1 < 0 ? -(d + 1) : d + 1));
}

// Summary of one 32-position block from its valid (V) and hit (H) masks
// (bit i = position i; H a subset of V). The gaps closed inside the block
// are walked one by one: from the first remaining valid miss after the first
// hit to the next hit.
IBS_HD Seg32 block_seg32(uint32_t V, uint32_t H, int k)
{
    Seg32 r;
    r.total = popc32(V);
    r.obs = popc32(H);
    r.gaps = 0;
    r.dist = 0;
    if (H == 0) {
        r.lead = r.trail = r.total;
        return r;
    }
    const uint32_t first = ctz32(H), last = 31 - clz32(H);
    r.lead = popc32(V & ((1u << first) - 1u));
    r.trail = popc32((V >> last) >> 1);
    // valid misses strictly between the first and the last hit (last > first
    // whenever there are any, so both shifts stay below 32)
    uint32_t M = last > first ? V & ~H & ((1u << last) - 1u) & ~((2u << first) - 1u) : 0u;
    while (M) {
        const uint32_t a = ctz32(M);                         // a < last
        const uint32_t nh = ctz32(H & ~((2u << a) - 1u));   // the hit that ends the gap
        const uint32_t below = (1u << nh) - 1u;
        const uint32_t g = popc32(M & below);
        r.gaps += 1;
        r.dist += gap_distance32(g, k);
        M &= ~below;
    }
    return r;
}

// a followed by b, without branches: a side without hits has lead == trail
// == total, and the gap across the boundary closes only between two hits.
IBS_HD Seg32 seg32_combine(const Seg32 &a, const Seg32 &b, int k)
{
    Seg32 r;
    r.total = a.total + b.total;
    r.obs = a.obs + b.obs;
    r.lead = a.obs ? a.lead : a.lead + b.lead;
    r.trail = b.obs ? b.trail : a.trail + b.trail;
    const uint32_t g = a.trail + b.lead;
    const bool close = a.obs && b.obs && g;
    r.gaps = a.gaps + b.gaps + (close ? 1u : 0u);
    r.dist = a.dist + b.dist + (close ? gap_distance32(g, k) : 0u);
    return r;
}

IBS_HD SegStats seg_of(const Seg32 &s)
{
    SegStats r;
    r.total = s.total;
    r.obs = s.obs;
    r.lead = s.lead;
    r.trail = s.trail;
    r.gaps = s.gaps;
    r.pad = 0;
    r.dist = s.dist;
    return r;
}

IBS_HD void seg_finish(const SegStats &s, int k, WindowRow &row)
{
    int64_t var = s.gaps, dist = s.dist;
    if (s.obs == 0) {
        if (s.total > 0) {
            var += 1;
            dist += gap_distance(s.total, k);
        }
    } else {
        if (s.lead > 0) {
            var += 1;
            dist += gap_distance(s.lead, k);
        }
        if (s.trail > 0) {
            var += 1;
            dist += gap_distance(s.trail, k);
        }
    }
    row.total_kmers = (int32_t)s.total;
    row.observed_kmers = (int32_t)s.obs;
    row.variations = (int32_t)var;
    row.kmer_distance = (int32_t)dist;
}

// ---------------------------------------------------------------------------
// Windowing: chunkSequences (src/Utils.hpp:296-327) cuts [j, min(j+W, len))
// for j = 0, W-k, 2(W-k), ... while j < len; a window has max(0, n-k+1)
// k-mer positions.
// ---------------------------------------------------------------------------
IBS_HD uint64_t windows_in_contig(uint64_t len, uint32_t W, uint32_t k)
{
    const uint64_t step = (uint64_t)W - k;
    return len ? (len + step - 1) / step : 0;
}

// ---------------------------------------------------------------------------
// 2-bit reference packing, the reference's packWindow convention
// (src/gpu/EncodeProbeCore.hpp:157-186) applied to a whole contig: base b
// at bits 2(b%32) of u64 word b/32 (A=0 C=1 G=2 T=3), and bit b%64 of u64
// mask word b/64 set when the byte is not ACGT/acgt. Contig c starts at
// packed base offset sum_{c'<c} roundup64(len_c'), so every contig begins
// on a mask-word boundary; both arrays carry one zero word of tail padding.
// ---------------------------------------------------------------------------
IBS_HD uint64_t round_up64(uint64_t x) { return (x + 63) & ~63ull; }

} // namespace ibs
