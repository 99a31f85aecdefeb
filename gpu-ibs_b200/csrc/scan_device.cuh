// Device helpers of the window scan: the 32-position block statistics from
// hit/valid ballots and the canonical code of a k-mer read from the 2-bit
// packed reference. See ibs_scan.cu for the kernel they serve.
#pragma once

#include "ibs_core.cuh"

namespace ibs {
namespace dev {

constexpr uint32_t FULL_MASK = 0xffffffffu;

// Statistics of one 32-position block from its valid (V) and hit (H)
// ballots (bit i = position p+i; H is a subset of V); every lane returns the
// same value. The lane of each hit except the first counts the valid misses
// since the previous hit, so the gaps closed inside the block are found
// lane-parallel.
__device__ __forceinline__ SegStats block_stats(uint32_t V, uint32_t H, uint32_t lane, int k)
{
    SegStats b;
    b.pad = 0;
    b.total = __popc(V);
    b.obs = __popc(H);
    if (H == 0) {
        b.lead = b.trail = b.total;
        b.gaps = 0;
        b.dist = 0;
        return b;
    }
    const uint32_t first = __ffs(H) - 1;
    const uint32_t last = 31 - __clz(H);
    b.lead = __popc(V & ((1u << first) - 1u));
    b.trail = last == 31 ? 0u : __popc(V >> (last + 1));
    uint32_t g = 0;
    if (((H >> lane) & 1u) && lane != first) {
        const uint32_t below = (1u << lane) - 1u;
        const uint32_t prev = 31 - __clz(H & below);
        g = __popc(V & below & ~((2u << prev) - 1u));
    }
    const uint32_t gc = g > 0 ? 1u : 0u;
    const uint32_t d = g > 0 ? (uint32_t)gap_distance(g, k) : 0u;
    b.gaps = __reduce_add_sync(FULL_MASK, gc);
    b.dist = __reduce_add_sync(FULL_MASK, d);
    return b;
}

// Window statistics of a warp's span, folded 32 blocks at a time: lane i
// keeps the valid / hit ballots of the span's blocks i, i + 32, ...; after
// every 32 blocks (and at the end of the span) each lane summarises its own
// block with 32-bit operations and a shuffle tree combines the 32 summaries
// in block order into the running summary. A block costs the keeping lane a
// compare and two selects.
struct LaneFold {
    uint32_t v = 0, h = 0; // this lane's block since the last flush
    uint32_t n = 0;        // blocks since the last flush (warp-uniform)
    Seg32 acc{0, 0, 0, 0, 0, 0};

    __device__ __forceinline__ void push(uint32_t V, uint32_t H, uint32_t lane, int k)
    {
        if (lane == n) {
            v = V;
            h = H;
        }
        if (++n == 32)
            flush(k);
    }

    __device__ __forceinline__ void flush(int k)
    {
        Seg32 s = block_seg32(v, h, k); // lanes past n hold empty blocks
#pragma unroll
        for (uint32_t off = 1; off < 32; off <<= 1) {
            Seg32 o;
            o.total = __shfl_down_sync(FULL_MASK, s.total, off);
            o.obs = __shfl_down_sync(FULL_MASK, s.obs, off);
            o.lead = __shfl_down_sync(FULL_MASK, s.lead, off);
            o.trail = __shfl_down_sync(FULL_MASK, s.trail, off);
            o.gaps = __shfl_down_sync(FULL_MASK, s.gaps, off);
            o.dist = __shfl_down_sync(FULL_MASK, s.dist, off);
            s = seg32_combine(s, o, k); // right for lanes that are multiples of 2 off
        }
        acc = seg32_combine(acc, s, k); // lane 0's is the span so far
        v = h = n = 0;
    }

    // The span's summary (lane 0).
    __device__ __forceinline__ SegStats finish(int k)
    {
        if (n)
            flush(k);
        return seg_of(acc);
    }
};

// Canonical code of the k-mer whose first base is packed base G, and whether
// its k bases are all ACGT. Reads two sequence words and two mask words.
__device__ __forceinline__ uint64_t canonical_at(const uint64_t *__restrict__ seq,
                                                 const uint64_t *__restrict__ mask, uint64_t G,
                                                 uint32_t k, uint64_t kmask, uint64_t kbits,
                                                 bool &acgt)
{
    const uint64_t wi = G >> 5;
    const uint32_t sh = (uint32_t)(G & 31) * 2;
    const uint64_t w0 = __ldg(seq + wi), w1 = __ldg(seq + wi + 1);
    const uint64_t x = (w0 >> sh) | ((w1 << (63 - sh)) << 1);
    const uint64_t mi = G >> 6;
    const uint32_t ms = (uint32_t)(G & 63);
    const uint64_t m0 = __ldg(mask + mi), m1 = __ldg(mask + mi + 1);
    const uint64_t mm = (m0 >> ms) | ((m1 << (63 - ms)) << 1);
    acgt = (mm & kbits) == 0;
    uint64_t y = __brevll(x);
    y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
    const uint64_t fwd = y >> (64 - 2 * k);
    const uint64_t rc = ~x & kmask;
    return fwd < rc ? fwd : rc;
}

} // namespace dev
} // namespace ibs
