// Host build of the window-statistics fold the scan kernel uses
// (gpu-ibs_b200/csrc/ibs_core.cuh), for property tests on the CPU.
#include <cstdint>
#include "ibs_core.cuh"

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
