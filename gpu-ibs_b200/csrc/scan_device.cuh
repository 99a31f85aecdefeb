// Device helpers of the window scans: the span statistics fold over
// hit/valid ballots and the canonical code of a k-mer read from the 2-bit
// packed reference. See ibs_scan.cu for the kernels they serve.
#pragma once

#include "ibs_core.cuh"

namespace ibs {
namespace dev {

constexpr uint32_t FULL_MASK = 0xffffffffu;

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
