// Host build of the window-statistics fold the scan kernel uses
// (gpu-ibs_b200/csrc/ibs_core.cuh), for property tests on the CPU.
#include <algorithm>
#include <cstdint>
#include "ibs_core.cuh"
#include "wide_core.cuh"

using namespace ibs;

// Folds positions [0, n) (valid[i], hit[i]) split into segments at the
// given cut points, combining segment summaries left to right, and returns
// the row values (total, observed, variations, distance).
extern "C" void fold_segments(const uint8_t *valid, const uint8_t *hit, uint64_t n,
                              const uint64_t *cuts, uint64_t nCuts, int k, int32_t out[4])
{
    SegStats acc = seg_empty();
    uint64_t a = 0;
    for (uint64_t c = 0; c <= nCuts; ++c) {
        const uint64_t b = c < nCuts ? cuts[c] : n;
        SegStats seg = seg_empty();
        for (uint64_t i = a; i < b; ++i) {
            SegStats one = seg_empty();
            if (valid[i]) {
                one.total = 1;
                if (hit[i])
                    one.obs = 1;
                else
                    one.lead = one.trail = 1;
            }
            seg = seg_combine(seg, one, k);
        }
        acc = seg_combine(acc, seg, k);
        a = b;
    }
    WindowRow row{};
    seg_finish(acc, k, row);
    out[0] = row.total_kmers;
    out[1] = row.observed_kmers;
    out[2] = row.variations;
    out[3] = row.kmer_distance;
}

// Bijectivity spot check of the table hash on a small key space.
extern "C" uint64_t hash_collisions(uint32_t bits)
{
    const uint64_t n = 1ull << bits;
    uint64_t coll = 0;
    uint8_t *seen = new uint8_t[n]();
    for (uint64_t x = 0; x < n; ++x) {
        const uint64_t h = perm_hash(x, bits);
        if (h >= n || seen[h]++)
            coll++;
    }
    delete[] seen;
    return coll;
}

// ---- minimizer-bucketed table (gpu-ibs_b200/csrc/mz_core.cuh) -------------
#include "mz_core.cuh"

static TableGeom mz_geom(uint32_t k, uint64_t nBuckets)
{
    TableGeom g{};
    g.k = k;
    g.bits = 2 * k;
    g.format = FMT_MZ8;
    g.nBuckets = nBuckets; // a multiple of the four sectors of a line
    g.fpBits = 2 * mz::m_of(k) - (63 - __builtin_clzll(nBuckets / mz::kSectorsPerLine));
    return g;
}

// Build side: bucket and slot of canonical codes.
extern "C" void mz_locate(const uint64_t *codes, uint64_t n, uint32_t k, uint64_t nBuckets,
                          uint64_t *bucket, uint64_t *slot)
{
    const TableGeom g = mz_geom(k, nBuckets);
    for (uint64_t i = 0; i < n; ++i)
        mz::locate(codes[i], g, bucket[i], slot[i]);
}

// Query side as the scan kernel computes it: along the forward strand of
// `bases` (values 0-3), m-mer rank keys per position, the window minimum over
// the next w keys with its leftmost/rightmost offsets, the strand of the
// canonical k-mer, then bucket and slot. Positions 0..n-k.
extern "C" void mz_query(const uint8_t *bases, uint64_t n, uint32_t k, uint64_t nBuckets,
                         uint64_t *bucket, uint64_t *slot)
{
    const TableGeom g = mz_geom(k, nBuckets);
    const uint32_t w = mz::w_of(k), m = mz::m_of(k);
    if (n < k)
        return;
    const uint64_t nm = n - m + 1;
    uint32_t *key = new uint32_t[nm];
    uint64_t *lg = new uint64_t[nm];   // line hash of the canonical m-mer
    uint8_t *fnc = new uint8_t[nm], *rnc = new uint8_t[nm]; // forward / its rc not canonical
    for (uint64_t q = 0; q < nm; ++q) {
        uint64_t f = 0, r = 0;
        for (uint32_t t = 0; t < m; ++t) {
            f = (f << 2) | bases[q + t];
            r |= (uint64_t)(3 - bases[q + t]) << (2 * t);
        }
        const uint64_t c = f < r ? f : r;
        key[q] = mz::rank_key(c, m);
        lg[q] = mz::line_hash(c, m);
        fnc[q] = f > r;
        rnc[q] = r > f;
    }
    const uint64_t kmask = key_mask(2 * k);
    for (uint64_t q = 0; q + k <= n; ++q) {
        uint64_t fwd = 0, rc = 0;
        for (uint32_t t = 0; t < k; ++t) {
            fwd = (fwd << 2) | bases[q + t];
            rc |= (uint64_t)(3 - bases[q + t]) << (2 * t);
        }
        rc &= kmask;
        const bool isFwd = fwd <= rc;
        const uint64_t C = isFwd ? fwd : rc;
        // the kernel's packed minimum: offset j (forward) or 7 - j (reverse)
        // in the keys' 3 clear low bits
        const uint32_t flip = isFwd ? 0u : 7u;
        uint32_t best = 0xffffffffu;
        for (uint32_t j = 0; j < w; ++j)
            best = std::min(best, key[q + j] ^ j ^ flip);
        const uint32_t jm = (best & 7u) ^ flip;
        const uint64_t src = q + jm;
        const uint32_t o = isFwd ? jm : (w - 1 - jm);
        mz::place(C, k, o, isFwd ? fnc[src] : rnc[src], lg[src], g.nBuckets, g.fpBits, bucket[q], slot[q]);
    }
    delete[] key;
    delete[] lg;
    delete[] fnc;
    delete[] rnc;
}

// The scan kernels' span fold (LaneFold, gpu-ibs_b200/csrc/scan_device.cuh)
// with its 32 lanes emulated: positions [0, n) in 32-position blocks, lane i
// keeping block i of every 32; each flush summarises the lanes' blocks
// (block_seg32) and combines them with the kernel's shuffle tree (lane l
// takes lane l + off's value, or its own past lane 31); then the row values.
extern "C" void span_fold(const uint8_t *valid, const uint8_t *hit, uint64_t n, int k, int32_t out[4])
{
    Seg32 acc{0, 0, 0, 0, 0, 0};
    uint32_t v[32] = {}, h[32] = {}, kept = 0;
    auto flush = [&]() {
        Seg32 s[32];
        for (int l = 0; l < 32; ++l)
            s[l] = block_seg32(v[l], h[l], k);
        for (int off = 1; off < 32; off <<= 1) {
            Seg32 t[32];
            for (int l = 0; l < 32; ++l)
                t[l] = seg32_combine(s[l], l + off < 32 ? s[l + off] : s[l], k);
            for (int l = 0; l < 32; ++l)
                s[l] = t[l];
        }
        acc = seg32_combine(acc, s[0], k);
        for (int l = 0; l < 32; ++l)
            v[l] = h[l] = 0;
        kept = 0;
    };
    for (uint64_t a = 0; a < n; a += 32) {
        uint32_t V = 0, H = 0;
        for (uint64_t i = a; i < n && i < a + 32; ++i) {
            V |= (uint32_t)(valid[i] != 0) << (i - a);
            H |= (uint32_t)(valid[i] && hit[i]) << (i - a);
        }
        v[kept] = V;
        h[kept] = H;
        if (++kept == 32)
            flush();
    }
    if (kept)
        flush();
    WindowRow row{};
    seg_finish(seg_of(acc), k, row);
    out[0] = row.total_kmers;
    out[1] = row.observed_kmers;
    out[2] = row.variations;
    out[3] = row.kmer_distance;
}

// Wide codes (wide_core.cuh): the canonical code and ACGT flag of the k-mer
// at each packed base G0 .. G0 + n - 1 of a packed reference (33 <= k <= 64),
// as the wide scan kernel reads them; lo / hi / ok get n entries.
extern "C" void wide_codes_packed(const uint64_t *seq, const uint64_t *mask, uint64_t G0, uint64_t n, uint32_t k,
                                  uint64_t *lo, uint64_t *hi, uint8_t *ok)
{
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t G = G0 + i;
        bool acgt = false;
        const uint64_t wi = G >> 5, mi = G >> 6;
        ibs::wide::canonical_from_words(seq[wi], seq[wi + 1], seq[wi + 2], mask[mi], mask[mi + 1], G, k, acgt,
                                        lo[i], hi[i]);
        ok[i] = acgt ? 1 : 0;
    }
}

// The wide table's line of a key in a level (wide_core.cuh), for the host
// tests of the level layout.
extern "C" uint64_t wide_line_of(uint64_t lo, uint64_t hi, uint32_t level, uint64_t lines)
{
    return ibs::wide::line_of(lo, hi, level, lines);
}
