// The minimizer-line scan of one span of positions, shared by the window
// scan (ibs_scan.cu) and the serving kernels (ibs_serve.cu).
//
// Each position's words are read once, one block ahead: the m-mer keys of
// the next block are needed by the current block's minimizer windows, and
// the same read gives the k-mer that block probes when its turn comes. A
// k-mer's minimizer is the minimum over the next w lanes' keys (shuffles
// across the block boundary); each key carries its offset j in its 3 low
// bits (j for a forward k-mer, 7 - j for a reverse one), so one integer
// minimum per offset keeps the leftmost-in-the-canonical-k-mer rule on either
// strand. Its line hash comes from the keying lane by shuffle. Lanes whose
// k-mers share a minimizer load sectors of one line.
#pragma once

#include "ibs_internal.cuh"
#include "scan_device.cuh"

namespace ibs {
namespace dev {

// Everything the minimizer scan needs about reference position G, from one
// read of its packed words: the canonical k-mer starting there (its code,
// strand and whether its k bases are all ACGT) and the m-mer starting there
// (its rank key, and its line hash with the orientation bits on top: bit 62
// set when the forward m-mer is not canonical, bit 63 when its reverse
// complement is not; 2m <= 42 leaves them free).
struct MzPos {
    uint64_t code, gs;
    uint32_t key;
    bool isFwd, acgt;
};

// The 32 bases from packed base G (bits 2t) and the N bits of the k from G,
// read as 32-bit words (base b at bits 2(b % 16) of word b / 16, N bit b at
// bit b % 32 of word b / 32) and joined by funnel shifts. The words read lie
// inside the 64-bit words G / 32 .. G / 32 + 1 and G / 64 .. G / 64 + 1.
__device__ __forceinline__ MzPos mz_pos(const uint64_t *__restrict__ seq, const uint64_t *__restrict__ mask,
                                        uint64_t G, uint32_t k, uint32_t m)
{
    MzPos r;
    const uint32_t *__restrict__ s32 = reinterpret_cast<const uint32_t *>(seq);
    const uint32_t *__restrict__ m32 = reinterpret_cast<const uint32_t *>(mask);
    const uint64_t wi = G >> 4;
    const uint32_t sh = (uint32_t)(G & 15) * 2;
    const uint32_t w0 = __ldg(s32 + wi), w1 = __ldg(s32 + wi + 1), w2 = __ldg(s32 + wi + 2);
    const uint64_t x = ((uint64_t)__funnelshift_r(w1, w2, sh) << 32) | __funnelshift_r(w0, w1, sh);
    const uint64_t mi = G >> 5;
    const uint32_t mm = __funnelshift_r(__ldg(m32 + mi), __ldg(m32 + mi + 1), (uint32_t)(G & 31));
    r.acgt = (mm & (uint32_t)key_mask(k)) == 0;
    uint64_t y = __brevll(x);
    y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1); // first base high
    const uint64_t fwd = y >> (64 - 2 * k);
    const uint64_t rc = ~x & key_mask(2 * k);
    r.isFwd = fwd <= rc;
    r.code = r.isFwd ? fwd : rc;
    const uint64_t f = y >> (64 - 2 * m);
    const uint64_t mr = ~x & key_mask(2 * m);
    const bool fLess = f < mr;
    const uint64_t c = fLess ? f : mr;
    const uint64_t lh = mz::line_hash(c, m);
    // an m-mer of odd length is never its own reverse complement (its middle
    // base would be its own complement), so one comparison gives both bits
    const uint64_t orient = (m & 1) ? (fLess ? 1ull << 63 : 1ull << 62)
                                    : ((f > mr ? 1ull << 62 : 0ull) | (fLess ? 1ull << 63 : 0ull));
    r.gs = lh | orient;
    r.key = mz::rank_key_of(lh);
    return r;
}

// Sector and slot value of this lane's k-mer (position q of a block) from
// the block's positions (cur) and the next block's (nxt): its minimizer is
// the smallest rank key over the w (<= 7) m-mers starting at q .. q+w-1,
// found with one shuffle per offset, and its line hash and orientation come
// from the keying lane.
// SLOT32: the table's slot values fit 32 bits (MZ8, joint minimizer lines).
template <bool SLOT32>
__device__ __forceinline__ void mz_locate_lane(const MzPos &cur, const MzPos &nxt, uint32_t lane, uint32_t k,
                                               uint32_t w, uint64_t nBuckets, uint32_t fpBits, uint64_t &r,
                                               uint64_t &slot)
{
    const bool isFwd = cur.isFwd;
    // keys have their low 3 bits clear; j ^ flip there makes the smallest
    // packed value the leftmost smallest key (forward k-mer) or the rightmost
    // (reverse k-mer)
    const uint32_t flip = isFwd ? 0u : 7u;
    uint32_t best = 0xffffffffu;
#pragma unroll
    for (uint32_t j = 0; j < 8; ++j) {
        if (j < w) {
            // key of position q + j: lanes below 32 - j read lane + j of this
            // block, the others lane + j - 32 (< j) of the next, so a source
            // lane offers its next-block key exactly when it is below j -- one
            // shuffle per offset
            const uint32_t offer = lane < j ? nxt.key : cur.key;
            const uint32_t v = __shfl_sync(FULL_MASK, offer, lane + j); // source lane mod 32
            best = min(best, v ^ j ^ flip);
        }
    }
    const uint32_t jm = (best & 7u) ^ flip;
    // the minimizer's line hash and orientation from the lane that keyed it:
    // position q + jm
    const uint32_t src = lane + jm;
    const uint64_t ga = __shfl_sync(FULL_MASK, cur.gs, src);
    const uint64_t gc = __shfl_sync(FULL_MASK, nxt.gs, src);
    const uint64_t gs = src < 32 ? ga : gc;
    const uint32_t sm = isFwd ? (uint32_t)(gs >> 62) & 1u : (uint32_t)(gs >> 63);
    const uint32_t o = isFwd ? jm : (w - 1 - jm);
    // place() and place32() read bits 0 .. 2m-1 of the line hash: the
    // orientation bits 62 and 63 above them need no masking
    if constexpr (SLOT32)
        mz::place32(cur.code, k, o, sm, gs, nBuckets, fpBits, r, slot);
    else
        mz::place(cur.code, k, o, sm, gs, nBuckets, fpBits, r, slot);
}

// Statistics of positions [p0, p1) of the window whose first base is packed
// base `base`, against a minimizer-line table; the m-mer reads stop at
// position lastM (the last m-mer start the window's k-mers use: lanes past
// the span read positions up to it, inside the window's bases, and are masked
// out). The result is in lane 0. K > 0 fixes k at compile time; K = 0 reads
// it from the table. SEC: FMT_B8X32 sectors (format MZ8) or FMT_B6X40 (MZ6).
template <int NB, uint32_t K, uint32_t SEC>
__device__ __forceinline__ SegStats mz_span_stats(const TableView &t, const uint64_t *__restrict__ seq,
                                                  const uint64_t *__restrict__ mask, uint64_t base, uint32_t p0,
                                                  uint32_t p1, uint32_t lastM, uint32_t lane)
{
    const uint32_t k = K ? K : t.g.k;
    const uint32_t w = mz::w_of(k);
    const uint32_t m = mz::m_of(k);
    LaneFold fold;
    MzPos next = mz_pos(seq, mask, base + min(p0 + lane, lastM), k, m);
    for (uint32_t p = p0; p < p1; p += 32 * NB) {
        MzPos ps[NB + 1];
        ps[0] = next;
#pragma unroll
        for (int b = 1; b <= NB; ++b)
            ps[b] = mz_pos(seq, mask, base + min(p + 32 * b + lane, lastM), k, m);
        next = ps[NB];
        uint4 v0[NB], v1[NB];
        uint64_t slot[NB], rb[NB];
        bool valid[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const uint32_t q = p + 32 * b + lane;
            valid[b] = q < p1 && ps[b].acgt;
            uint64_t &r = rb[b];
            mz_locate_lane<false>(ps[b], ps[b + 1], lane, k, w, t.g.nBuckets, t.g.fpBits, r, slot[b]);
            if (valid[b]) {
                v0[b] = __ldg(t.buckets + 2 * r);
                v1[b] = __ldg(t.buckets + 2 * r + 1);
            } else {
                v0[b] = make_uint4(0, 0, 0, 0);
                v1[b] = make_uint4(0, 0, 0, 0);
            }
        }
        uint32_t V[NB], H[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            bool hit = false;
            if (valid[b]) {
                if constexpr (SEC == FMT_B8X32) {
                    const uint32_t mt = mz8_match(v0[b], v1[b], (uint32_t)slot[b]);
                    hit = mt == 1u ||
                          (mt >= 2u && mz8_overflow_lookup(t, rb[b], (uint32_t)slot[b], mt, ps[b].code));
                } else {
                    const uint32_t mt = bucket_match<SEC>(v0[b], v1[b], slot[b]);
                    hit = mt == 1u || (mt == 2u && stash_lookup(t, ps[b].code));
                }
            }
            V[b] = __ballot_sync(FULL_MASK, valid[b]);
            H[b] = __ballot_sync(FULL_MASK, hit);
        }
#pragma unroll
        for (int b = 0; b < NB; ++b)
            fold.push(V[b], H[b], lane, (int)k);
    }
    return fold.finish((int)k);
}

} // namespace dev
} // namespace ibs
