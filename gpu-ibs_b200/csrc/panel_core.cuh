// Panel scan: one reference pass against up to 16 samples through ONE joint
// table whose slots carry a sample-membership mask.
//
// The reference's panel mode encodes each batch once and probes every
// resident database separately (encodeProbeMultiKernel + MultiBsProbe,
// src/gpu/EncodeProbe.cu:82-108, :175-193; MAX_DBS = 16,
// src/gpu/EncodeProbeCore.hpp:291), so a position costs one index search
// per sample. Here the samples' k-mer sets are merged into one table: a
// position costs one random 32-byte bucket load whatever the panel size,
// and the mask in the matching slot says which samples hold the k-mer.
// Every sample's rows are still exactly its single-sample rows.
//
// Bucket format P5x48 (one 32-byte sector): u32 fingerprints of slots 0-4
// (words 0-4), u16 sample masks of slots 0-4 (bytes 20-29), slot count
// (byte 30), flags (byte 31, bit 0 = some key of this bucket is in the
// stash). The fingerprint is the same quotient of the bijective k-mer hash
// as in the single-sample table, so it needs nBuckets >= 2^(2k-32).
// Stash: {code, mask} pairs, two per 32-byte bucket, linear probing.
//
// Format PM (FMT_PANEL_MZ, 16 <= k <= 27): the same sectors laid out as the
// minimizer lines of the single-sample MZ tables (mz_core.cuh): the line is
// the k-mer's minimizer's, one of its four sectors is picked by the k-mer
// itself, and the 32-bit slot value identifies the k-mer within its line
// (at least 2^(2k-28) lines). Consecutive reference positions mostly share a
// minimizer, so a warp's probes fall in few 128-byte lines instead of 32
// random ones. A full sector keeps further keys in its partner sector (index
// ^ 1, the same line; flag bit 25 of byte 31's word) and then in the stash
// (bit 24).
#pragma once

#include "ibs_internal.cuh"
#include "mz_core.cuh"

#include <vector>

namespace ibs {
namespace panel {

constexpr uint32_t kMaxSamples = IBS_PANEL_MAX_SAMPLES;
constexpr uint32_t kSlots = 5;
constexpr uint64_t kStashEmpty = ~0ull;
constexpr uint32_t kStashFlag = 1u << 24;   // word 7: some key of this sector is in the stash
constexpr uint32_t kPartnerFlag = 1u << 25; // word 7 (PM): some key of this sector is in its partner sector

struct View {
    TableGeom g;
    const uint4 *buckets;
    const ulonglong2 *stash; // {code, mask}
    uint64_t stashBuckets;   // power of two; two entries each
};

__device__ __forceinline__ uint32_t stash_mask(const View &t, uint64_t code)
{
    uint64_t b = stash_home(code, t.stashBuckets);
    for (uint64_t i = 0; i < t.stashBuckets; ++i) {
        const ulonglong2 e0 = __ldg(t.stash + 2 * b), e1 = __ldg(t.stash + 2 * b + 1);
        if (e0.x == code)
            return (uint32_t)e0.y;
        if (e1.x == code)
            return (uint32_t)e1.y;
        if (e0.x == kStashEmpty || e1.x == kStashEmpty)
            return 0;
        b = (b + 1) & (t.stashBuckets - 1);
    }
    return 0;
}

// Sample mask of fingerprint (or slot value) fp in a sector's halves; 0
// when no slot holds it.
__device__ __forceinline__ uint32_t sector_mask(const uint4 &v0, const uint4 &v1, uint32_t fp)
{
    const uint32_t cnt = (v1.w >> 16) & 0xff;
    uint32_t m = 0;
    m |= (0 < cnt && v0.x == fp) ? (v1.y & 0xffff) : 0u;
    m |= (1 < cnt && v0.y == fp) ? (v1.y >> 16) : 0u;
    m |= (2 < cnt && v0.z == fp) ? (v1.z & 0xffff) : 0u;
    m |= (3 < cnt && v0.w == fp) ? (v1.z >> 16) : 0u;
    m |= (4 < cnt && v1.x == fp) ? (v1.w & 0xffff) : 0u;
    return m;
}

// Sample mask of a k-mer given its bucket halves and fingerprint; bit 31
// set = look in the stash.
__device__ __forceinline__ uint32_t bucket_mask(const uint4 &v0, const uint4 &v1, uint32_t fp)
{
    uint32_t m = sector_mask(v0, v1, fp);
    if (!m && (v1.w & kStashFlag))
        m = 0x80000000u;
    return m;
}

// PM: the mask of the k-mer `code` with slot value `slot` whose home
// sector r has halves v0, v1: the home sector, then (flagged) its partner
// sector, then (flagged) the stash.
__device__ __forceinline__ uint32_t pm_mask(const View &t, const uint4 &v0, const uint4 &v1, uint64_t r,
                                            uint32_t slot, uint64_t code)
{
    uint32_t m = sector_mask(v0, v1, slot);
    if (m)
        return m;
    if (v1.w & kPartnerFlag) {
        const uint4 w0 = __ldg(t.buckets + 2 * (r ^ 1)), w1 = __ldg(t.buckets + 2 * (r ^ 1) + 1);
        m = sector_mask(w0, w1, slot);
        if (m)
            return m;
    }
    return (v1.w & kStashFlag) ? stash_mask(t, code) : 0u;
}

// Home sector and stored fingerprint (P5x48) or slot value (PM) of a key.
__device__ __forceinline__ void joint_place(const View &t, uint64_t code, uint64_t &r, uint32_t &fp)
{
    if (t.g.format == FMT_PANEL_MZ) {
        uint64_t slot;
        mz::locate(code, t.g, r, slot);
        fp = (uint32_t)slot;
        return;
    }
    const uint64_t h = perm_hash(code, t.g.bits);
    r = bucket_of(h, t.g);
    fp = (uint32_t)fp_of(h, t.g);
}

__device__ __forceinline__ uint32_t lookup_mask(const View &t, uint64_t code)
{
    if (t.g.format == FMT_PANEL_MZ) {
        uint64_t r;
        uint32_t slot;
        joint_place(t, code, r, slot);
        const uint4 v0 = __ldg(t.buckets + 2 * r), v1 = __ldg(t.buckets + 2 * r + 1);
        return pm_mask(t, v0, v1, r, slot, code);
    }
    const uint64_t h = perm_hash(code, t.g.bits);
    const uint64_t r = bucket_of(h, t.g);
    const uint4 v0 = __ldg(t.buckets + 2 * r), v1 = __ldg(t.buckets + 2 * r + 1);
    uint32_t m = bucket_mask(v0, v1, (uint32_t)fp_of(h, t.g));
    if (m & 0x80000000u)
        m = stash_mask(t, code);
    return m;
}

// Block statistics of one sample from its valid (V) and hit (H) masks,
// computed by one lane with bit operations: the gaps between hits are the
// runs of valid misses, visited one run at a time.
__device__ __forceinline__ SegStats block_stats_serial(uint32_t V, uint32_t H, int k)
{
    SegStats b;
    b.pad = 0;
    b.total = __popc(V);
    b.obs = __popc(H);
    b.gaps = 0;
    b.dist = 0;
    if (H == 0) {
        b.lead = b.trail = b.total;
        return b;
    }
    const uint32_t first = __ffs(H) - 1;
    const uint32_t last = 31 - __clz(H);
    b.lead = __popc(V & ((1u << first) - 1u));
    b.trail = last == 31 ? 0u : __popc(V >> (last + 1));
    // valid misses strictly between the first and the last hit
    const uint64_t inner = ((2ull << last) - 1ull) & ~((2ull << first) - 1ull);
    uint32_t m = V & ~H & (uint32_t)inner;
    while (m) {
        const uint32_t start = __ffs(m) - 1;
        const uint32_t next = H & ~((2u << start) - 1u); // hits after the run starts (nonzero)
        const uint32_t j = __ffs(next) - 1;
        const uint32_t g = __popc(m & ((1u << j) - 1u));
        b.gaps += 1;
        b.dist += gap_distance(g, k);
        m &= ~((1u << j) - 1u);
    }
    return b;
}

} // namespace panel
} // namespace ibs

// A joint table and its scan state (the handle behind the ibs_panel_table_* calls).
struct ibs_panel_table {
    using View = ibs::panel::View;
    int device = 0;
    ibs::TableGeom geom{};
    uint4 *buckets = nullptr;
    ulonglong2 *stash = nullptr;
    uint64_t stashBuckets = 0;
    uint32_t nSamples = 0;
    uint64_t keysAdded = 0; // sum of the samples' key counts
    uint64_t deviceBytes = 0;
    double buildSeconds = 0;
    int *dErr = nullptr;
    unsigned long long *dCounters = nullptr; // [0] pending count, [1] scan work counter, [2] failed
    uint32_t stashGrowths = 0;
    // scan plan and scratch
    const ibs_reference *planRef = nullptr;
    std::vector<uint64_t> planLens;
    ibs::ScanPlan plan;
    ibs::SegStats *dSpans = nullptr;
    uint16_t *dMasks = nullptr; // per-position masks of a multi-pass scan
    uint64_t spansCap = 0;
    // captured scan graph for (reference, W, rows, stream)
    cudaGraphExec_t graph = nullptr;
    const void *graphKey[3] = {nullptr, nullptr, nullptr};
    uint32_t graphShape[3] = {0, 0, 0}; // what it was captured with: CTAs per SM, blocks in flight, passes
    uint32_t graphW = 0;
    View view() const { return View{geom, buckets, stash, stashBuckets}; }
};

namespace ibs {
void panel_release_table(ibs_panel_table *p);
} // namespace ibs
