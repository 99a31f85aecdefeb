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
enum : uint32_t { FMT_B8X32 = 1, FMT_B6X40 = 2, FMT_PANEL = 3, FMT_MZ8 = 4, FMT_AUTO_HASH = 5, FMT_MZ6 = 6 };
// Minimizer-line tables: B8x32 sectors (31-bit slot values) or B6x40 sectors
// (40-bit slot values, for larger k).
IBS_HD bool is_mz(uint32_t fmt) { return fmt == FMT_MZ8 || fmt == FMT_MZ6; }
constexpr uint32_t B8_EMPTY = 0xffffffffu;
constexpr uint32_t B8_OVERFLOW = 0xfffffffeu;
constexpr uint64_t STASH_EMPTY = ~0ull;

struct TableGeom {
    uint32_t k;        // k-mer length (<= 32)
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

IBS_HD uint32_t popc64(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return __popcll(x);
#else
    return (uint32_t)__builtin_popcountll(x);
#endif
}

// Index of the lowest / highest set bit of x != 0.
IBS_HD uint32_t ctz64(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return __ffsll(x) - 1;
#else
    return (uint32_t)__builtin_ctzll(x);
#endif
}

IBS_HD uint32_t clz64(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return __clzll(x);
#else
    return (uint32_t)__builtin_clzll(x);
#endif
}

// Running statistics of one warp's span, fed 64 positions at a time as
// valid (V) and hit (H) masks (bit i = the i-th position; H a subset of V).
// The counts, the misses before the span's first hit (lead) and since its
// last hit (pending) are warp-uniform. Gaps are closed where they end: a gap
// that ends at a chunk's first hit by every lane alike (lane 0 counts it), a
// gap inside a chunk by the lane of the hit that ends it. Each lane keeps its
// own gap sums; the warp adds them up once at the end of the span. Chunks
// with no valid miss between their first and last hit skip the per-lane
// search.
struct SpanFold {
    uint32_t total = 0, obs = 0, lead = 0, pending = 0;
    uint32_t gc = 0, d = 0; // this lane's closed gaps and their distance sum

    IBS_HD void add(uint64_t V, uint64_t H, uint32_t lane, int k)
    {
        const uint32_t nV = popc64(V);
        total += nV;
        if (H == 0) {
            if (obs == 0)
                lead += nV;
            else
                pending += nV;
            return;
        }
        const uint32_t first = ctz64(H);
        const uint32_t last = 63 - clz64(H);
        const uint32_t c0 = popc64(V & ((1ull << first) - 1ull));
        if (obs == 0) {
            lead += c0;
        } else if (pending + c0 > 0 && lane == 0) {
            gc += 1;
            d += (uint32_t)gap_distance(pending + c0, k);
        }
        obs += popc64(H);
        // valid misses strictly between the first and the last hit
        const uint64_t inner = V & ~H & ~((2ull << first) - 1ull) & ((1ull << last) - 1ull);
        if (inner) {
            for (uint32_t half = 0; half < 2; ++half) {
                const uint32_t pos = lane + 32 * half;
                if (((H >> pos) & 1ull) && pos != first) {
                    const uint64_t below = (1ull << pos) - 1ull;
                    const uint32_t prev = 63 - clz64(H & below); // a hit before pos
                    const uint32_t g = popc64(V & below & ~((2ull << prev) - 1ull));
                    if (g) {
                        gc += 1;
                        d += (uint32_t)gap_distance(g, k);
                    }
                }
            }
        }
        pending = last == 63 ? 0u : popc64(V >> (last + 1));
    }

    // The span's summary, given the sums of gc and d over the warp's lanes.
    IBS_HD SegStats summary(uint32_t gaps, uint32_t dist) const
    {
        SegStats r;
        r.pad = 0;
        r.total = total;
        r.obs = obs;
        r.lead = obs ? lead : total;
        r.trail = obs ? pending : total;
        r.gaps = gaps;
        r.dist = dist;
        return r;
    }
};

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
