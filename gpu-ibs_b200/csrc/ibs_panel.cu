// Panel scan over the joint table of panel_core.cuh: build (two-phase
// insertion per sample), the persistent span kernel and its CUDA graph, and
// the ibs_panel_table_* entry points.
#include "mz_scan.cuh"
#include "panel_core.cuh"
#include "scan_device.cuh"

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>

namespace ibs {
namespace panel {

// Stash buckets an insert looks at before it fails (the stash then grows).
constexpr uint64_t kStashProbe = 64;

// Default load of joint minimizer-line tables: keys per 5-slot sector (the
// keys of one minimizer crowd its line, so the load stays below the hash
// sectors' 3)
constexpr double kPmKeysPerSector = 1.5;
constexpr uint64_t kBuildChunk = 1ull << 27; // keys per build step (1 GiB of scratch each way)

// Slot of fingerprint fp among sector w's first count slots, or -1.
__device__ __forceinline__ int find_slot(const uint32_t *w, uint32_t fp)
{
    const uint32_t cnt = (w[7] >> 16) & 0xff;
    int slot = -1;
    for (uint32_t j = 0; j < cnt && j < kSlots; ++j)
        if (w[j] == fp)
            slot = (int)j;
    return slot;
}

// ORs `bit` into the stash entry of `code`; false when the stash lacks it.
__device__ __forceinline__ bool stash_or(const View &t, unsigned long long *stashWords, uint64_t code,
                                         uint32_t bit)
{
    uint64_t b = stash_home(code, t.stashBuckets);
    for (uint64_t s = 0; s < t.stashBuckets; ++s) {
        unsigned long long *e = stashWords + 4 * b;
        if (e[0] == code) {
            atomicOr(e + 1, 1ull << bit);
            return true;
        }
        if (e[2] == code) {
            atomicOr(e + 3, 1ull << bit);
            return true;
        }
        if (e[0] == kStashEmpty || e[2] == kStashEmpty)
            return false;
        b = (b + 1) & (t.stashBuckets - 1);
    }
    return false;
}

// Claims a free slot of sector w (bumps its count byte below kSlots) and
// fills it with fp and the sample bit; false when the sector is full.
__device__ __forceinline__ bool claim_slot(uint32_t *w, uint32_t fp, uint32_t bit)
{
    uint32_t old = w[7], slot = kSlots;
    for (int tries = 0; tries < 1 << 20; ++tries) {
        const uint32_t cnt = (old >> 16) & 0xff;
        if (cnt >= kSlots)
            break;
        const uint32_t seen = atomicCAS(w + 7, old, old + (1u << 16));
        if (seen == old) {
            slot = cnt;
            break;
        }
        old = seen;
    }
    if (slot >= kSlots)
        return false;
    w[slot] = fp;
    atomicOr(w + 5 + slot / 2, (1u << bit) << (16 * (slot & 1)));
    return true;
}

// ---- build: phase A finds keys already present and ORs in the sample bit;
// phase B inserts the rest. Within one sample the keys are unique, so no
// lookup races with an insert of the same key. A key is looked for where
// phase B would have put it: its home sector, then (PM, flagged) the home's
// partner sector, then (flagged) the stash.
__global__ void k_find(View t, uint32_t *words, unsigned long long *stashWords, const uint64_t *codes,
                       uint64_t n, uint32_t bit, uint64_t *pending, unsigned long long *nPending)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t iters = (n + stride - 1) / stride;
    const bool pm = t.g.format == FMT_PANEL_MZ;
    for (uint64_t it = 0; it < iters; ++it) {
        const uint64_t i = it * stride + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
        bool miss = false;
        uint64_t code = 0;
        if (i < n) {
            code = codes[i];
            uint64_t r;
            uint32_t fp;
            joint_place(t, code, r, fp);
            uint32_t *w = words + 8 * r;
            const uint32_t flags = w[7];
            int slot = find_slot(w, fp);
            uint32_t *where = w;
            if (slot < 0 && pm && (flags & kPartnerFlag)) {
                where = words + 8 * (r ^ 1);
                slot = find_slot(where, fp);
            }
            if (slot >= 0)
                atomicOr(where + 5 + slot / 2, (1u << bit) << (16 * (slot & 1)));
            else
                miss = !((flags & kStashFlag) && stash_or(t, stashWords, code, bit));
        }
        const uint32_t ballot = __ballot_sync(0xffffffffu, miss);
        if (!ballot)
            continue;
        unsigned long long base = 0;
        if (lane == 0)
            base = atomicAdd(nPending, (unsigned long long)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (miss)
            pending[base + __popc(ballot & ((1u << lane) - 1u))] = code;
    }
}

__global__ void k_insert(View t, uint32_t *words, unsigned long long *stashWords, const uint64_t *codes,
                         uint64_t n, uint32_t bit, uint64_t *failed, unsigned long long *nFailed)
{
    const bool pm = t.g.format == FMT_PANEL_MZ;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t code = codes[i];
        uint64_t r;
        uint32_t fp;
        joint_place(t, code, r, fp);
        uint32_t *w = words + 8 * r;
        if (claim_slot(w, fp, bit))
            continue;
        if (pm) { // the partner sector of the same line, flagged on the home sector
            atomicOr(w + 7, kPartnerFlag);
            if (claim_slot(words + 8 * (r ^ 1), fp, bit))
                continue;
        }
        atomicOr(w + 7, kStashFlag);
        uint64_t b = stash_home(code, t.stashBuckets);
        bool placed = false;
        // at most kStashProbe buckets from home: a crowded stash fails the
        // insert (the host doubles it and inserts again) instead of costing a
        // scan of the whole stash per key; lookups still stop at the first
        // empty entry, which lies beyond every key placed this way
        const uint64_t probes = t.stashBuckets < kStashProbe ? t.stashBuckets : kStashProbe;
        for (uint64_t s = 0; s < probes && !placed; ++s) {
            for (int e = 0; e < 2 && !placed; ++e) {
                unsigned long long *entry = stashWords + 4 * b + 2 * e;
                const unsigned long long prev = atomicCAS(entry, kStashEmpty, (unsigned long long)code);
                if (prev == kStashEmpty || prev == code) {
                    atomicOr(entry + 1, 1ull << bit);
                    placed = true;
                }
            }
            b = (b + 1) & (t.stashBuckets - 1);
        }
        if (!placed) // the stash is full: the host grows it and inserts these again
            failed[atomicAdd(nFailed, 1ull)] = code;
    }
}

// Moves every stash entry into a larger stash (the build's stash growth).
__global__ void k_stash_move(const ulonglong2 *old, uint64_t oldEntries, unsigned long long *fresh,
                             uint64_t freshBuckets, int *err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < oldEntries;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 e = old[i];
        if (e.x == kStashEmpty)
            continue;
        uint64_t b = stash_home(e.x, freshBuckets);
        bool placed = false;
        for (uint64_t s = 0; s < freshBuckets && !placed; ++s) {
            for (int j = 0; j < 2 && !placed; ++j) {
                unsigned long long *entry = fresh + 4 * b + 2 * j;
                if (atomicCAS(entry, kStashEmpty, (unsigned long long)e.x) == kStashEmpty) {
                    entry[1] = e.y;
                    placed = true;
                }
            }
            b = (b + 1) & (freshBuckets - 1);
        }
        if (!placed)
            atomicExch(err, 1);
    }
}

// The span kernel in three modes. kScan: probe and fold every sample's
// statistics (one pass). kMaskPass: probe only k-mers whose bucket lies in
// [bLo, bHi) and store (first pass) or OR in (later passes) their sample
// masks, 16 bits per position, into `masks`. kStats: fold the statistics
// from the stored masks. A joint table far larger than the GPU's address
// translation reach probes much slower at random; cutting its buckets into
// ranges probed in separate passes keeps each pass's random loads inside
// one range.
enum : int { kScan = 0, kMaskPass = 1, kStats = 2 };

template <int NB, int MODE, bool PM>
__global__ void __launch_bounds__(256) k_panel_spans(View t, const uint64_t *__restrict__ seq,
                                                     const uint64_t *__restrict__ mask,
                                                     const WinDesc *__restrict__ win,
                                                     const uint32_t *__restrict__ span0, uint32_t nWin,
                                                     uint64_t nSpans, uint32_t spanLen,
                                                     uint32_t nSamples,
                                                     unsigned long long *__restrict__ work,
                                                     SegStats *__restrict__ out, uint16_t *__restrict__ masks,
                                                     uint64_t bLo, uint64_t bHi, bool firstPass)
{
    // PM tables locate a k-mer through its minimizer (one block of m-mers
    // read ahead); the statistics pass only needs each position's validity
    constexpr bool kMz = PM && MODE != kStats;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t k = t.g.k;
    const uint64_t kmask = key_mask(2 * k);
    const uint64_t kbits = (1ull << k) - 1;
    const uint32_t w = kMz ? mz::w_of(k) : 1, m = kMz ? mz::m_of(k) : 0;
    for (;;) {
        unsigned long long s = 0;
        if (lane == 0)
            s = atomicAdd(work, 1ull);
        s = __shfl_sync(dev::FULL_MASK, s, 0);
        if (s >= nSpans)
            break;
        uint32_t lo = 0, hi = nWin - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(span0 + mid) <= s)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint64_t base = win[lo].base;
        const uint32_t nPos = win[lo].nPos;
        const uint32_t p0 = (uint32_t)(s - __ldg(span0 + lo)) * spanLen;
        const uint32_t p1 = min(p0 + spanLen, nPos);
        uint16_t *spanMasks = masks + s * spanLen - p0; // position q of the span at spanMasks[q]
        SegStats acc = seg_empty(); // lane j < nSamples: sample j
        // PM: the last m-mer start the window's k-mers use; lanes past the
        // span read up to it (inside the window's bases) and are masked out
        const uint32_t lastM = nPos - 1 + (w - 1);
        dev::MzPos next;
        if constexpr (kMz)
            next = dev::mz_pos(seq, mask, base + min(p0 + lane, lastM), k, m);
        for (uint32_t p = p0; p < p1; p += 32 * NB) {
            uint4 v0[NB], v1[NB];
            uint64_t code[NB], rr[NB];
            uint32_t fp[NB];
            bool valid[NB], mine[NB];
            if constexpr (kMz) {
                dev::MzPos ps[NB + 1];
                ps[0] = next;
#pragma unroll
                for (int b = 1; b <= NB; ++b)
                    ps[b] = dev::mz_pos(seq, mask, base + min(p + 32 * b + lane, lastM), k, m);
                next = ps[NB];
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    const uint32_t q = p + 32 * b + lane;
                    valid[b] = q < p1 && ps[b].acgt;
                    uint64_t slot;
                    dev::mz_locate_lane<true>(ps[b], ps[b + 1], lane, k, w, t.g.nBuckets, t.g.fpBits, rr[b], slot);
                    fp[b] = (uint32_t)slot;
                    code[b] = ps[b].code;
                }
            } else {
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    const uint32_t q = p + 32 * b + lane;
                    const bool inSpan = q < p1;
                    const uint64_t G = base + (inSpan ? q : p0);
                    bool acgt;
                    code[b] = dev::canonical_at(seq, mask, G, k, kmask, kbits, acgt);
                    valid[b] = inSpan && acgt;
                    const uint64_t h = perm_hash(code[b], t.g.bits);
                    rr[b] = bucket_of(h, t.g);
                    fp[b] = (uint32_t)fp_of(h, t.g);
                }
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                mine[b] = valid[b] && (MODE != kMaskPass || (rr[b] >= bLo && rr[b] < bHi));
                if (MODE != kStats && mine[b]) {
                    v0[b] = __ldg(t.buckets + 2 * rr[b]);
                    v1[b] = __ldg(t.buckets + 2 * rr[b] + 1);
                } else {
                    v0[b] = make_uint4(0, 0, 0, 0);
                    v1[b] = make_uint4(0, 0, 0, 0);
                }
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const uint32_t q = p + 32 * b + lane;
                uint32_t m = 0;
                if (MODE == kStats) {
                    if (valid[b])
                        m = spanMasks[q];
                } else if (mine[b]) {
                    if constexpr (kMz) {
                        m = pm_mask(t, v0[b], v1[b], rr[b], fp[b], code[b]);
                    } else {
                        m = bucket_mask(v0[b], v1[b], fp[b]);
                        if (m & 0x80000000u)
                            m = stash_mask(t, code[b]);
                    }
                }
                if (MODE == kMaskPass) {
                    if (q < p1 && (firstPass || m))
                        spanMasks[q] = (uint16_t)(firstPass ? m : (spanMasks[q] | m));
                    continue;
                }
                const uint32_t V = __ballot_sync(dev::FULL_MASK, valid[b]);
                uint32_t myH = 0;
                for (uint32_t j = 0; j < nSamples; ++j) {
                    const uint32_t Hj = __ballot_sync(dev::FULL_MASK, (m >> j) & 1u);
                    if (lane == j)
                        myH = Hj;
                }
                if (lane < nSamples)
                    acc = seg_combine(acc, block_stats_serial(V, myH, (int)k), (int)k);
            }
        }
        if (MODE != kMaskPass && lane < nSamples)
            out[(uint64_t)lane * nSpans + s] = acc;
    }
}

__global__ void k_panel_finalize(const WinDesc *__restrict__ win, const uint32_t *__restrict__ span0,
                                 uint64_t nWin, uint64_t nSpans, uint32_t nSamples,
                                 const SegStats *__restrict__ spans, int k, ibs_window *__restrict__ rows)
{
    const uint64_t total = nWin * nSamples;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t smp = x / nWin, w = x - smp * nWin;
        SegStats acc = seg_empty();
        for (uint32_t s = span0[w]; s < span0[w + 1]; ++s)
            acc = seg_combine(acc, spans[smp * nSpans + s], k);
        WindowRow row;
        row.start = win[w].start;
        row.end = win[w].end;
        seg_finish(acc, k, row);
        ibs_window o;
        o.start = row.start;
        o.end = row.end;
        o.total_kmers = row.total_kmers;
        o.observed_kmers = row.observed_kmers;
        o.variations = row.variations;
        o.kmer_distance = row.kmer_distance;
        rows[x] = o;
    }
}

// Empty stash: every entry {EMPTY, no samples}.
__global__ void k_stash_init(ulonglong2 *stash, uint64_t entries)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < entries;
         i += (uint64_t)gridDim.x * blockDim.x)
        stash[i] = make_ulonglong2(kStashEmpty, 0ull);
}

__global__ void k_probe_masks(View t, const uint64_t *codes, uint64_t n, uint32_t *masks)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        masks[i] = lookup_mask(t, codes[i]);
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

int grid_for(uint64_t n)
{
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 16));
}

// Expected fraction of keys beyond a bucket's kSlots slots when the keys per
// bucket are Poisson(lam).
double overflow_fraction(double lam)
{
    if (lam <= 0)
        return 0;
    double p = std::exp(-lam), over = 0;
    for (int x = 0; x < 400; ++x) {
        if (x > (int)kSlots)
            over += (x - (int)kSlots) * p;
        p *= lam / (x + 1);
    }
    return over / lam;
}

uint64_t next_pow2(uint64_t x)
{
    uint64_t p = 1;
    while (p < x)
        p <<= 1;
    return p;
}

} // namespace panel
} // namespace ibs

using namespace ibs;
using namespace ibs::panel;


extern "C" ibs_status ibs_panel_table_create(uint32_t k, uint64_t expected_keys,
                                             const ibs_table_opts *opts, ibs_panel_table **out)
{
    clear_error();
    if (!out || k == 0 || k > 32) {
        set_error("ibs_panel_table_create: bad argument");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    const int dev = opts ? opts->device : 0;
    ibs_status s = check_device_ordinal(dev);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(dev);
    std::unique_ptr<ibs_panel_table> p(new ibs_panel_table);
    p->device = dev;
    TableGeom &g = p->geom;
    g.k = k;
    g.bits = 2 * k;
    uint32_t fmt = opts ? opts->force_format : 0;
    if (fmt != 0 && fmt != FMT_PANEL && fmt != FMT_PANEL_MZ) {
        set_error("ibs_panel_table_create: joint tables are format 3 (hash sectors) or 7 (minimizer lines)");
        return IBS_ERR_ARG;
    }
    if (fmt == FMT_PANEL_MZ && (k < 16 || k > 27)) {
        set_error("joint minimizer-line tables (format 7) need 16 <= k <= 27");
        return IBS_ERR_UNSUPPORTED;
    }
    // minimizer lines: 32-bit slot values need at least 2^(2k-28) lines
    const double lamPm = (opts && opts->keys_per_bucket > 0) ? opts->keys_per_bucket : kPmKeysPerSector;
    const uint64_t pmMinLines = 1ull << std::max<int>(0, 2 * (int)k - 28);
    const uint64_t pmLines = (uint64_t)((double)expected_keys / lamPm / mz::kSectorsPerLine) + 1;
    if (fmt == 0 && k >= 16 && k <= 27 && pmLines >= pmMinLines && pmLines < (1ull << 31))
        fmt = FMT_PANEL_MZ; // the default where its minimum size does not oversize the table
    if (fmt == 0)
        fmt = FMT_PANEL;
    g.format = fmt;
    uint64_t nb;
    double lam;
    if (fmt == FMT_PANEL_MZ) {
        lam = lamPm;
        const uint64_t nLines = std::min<uint64_t>(std::max(pmLines, pmMinLines), (1ull << 31) - 1);
        nb = nLines * mz::kSectorsPerLine;
        g.nBuckets = nb;
        g.fpBits = 2 * mz::m_of(k) - (uint32_t)(63 - __builtin_clzll(nLines));
    } else {
        lam = (opts && opts->keys_per_bucket > 0) ? opts->keys_per_bucket : tuning().panel_keys_per_bucket;
        nb = (uint64_t)((double)expected_keys / lam) + 1;
        const uint64_t minN = g.bits > 32 ? (1ull << (g.bits - 32)) : 1;
        nb = std::max(nb, minN);
        if (g.bits < 64)
            nb = std::min<uint64_t>(nb, 1ull << g.bits);
        g.nBuckets = nb;
        g.fpBits = (uint32_t)std::max<int>(1, (int)g.bits - (int)(63 - __builtin_clzll(nb)));
    }
    // keys per bucket are ~Poisson(expected / nBuckets); the stash holds the
    // expected overflow at <= 2/3 load (it grows during the build if needed)
    // minimizer lines: the keys of one minimizer crowd its line, so far more
    // than a Poisson share of them overflows (about 2% at 1.5 keys per
    // sector, 10% at 3); sized here for twice that, the stash grows if needed
    const double over = fmt == FMT_PANEL_MZ
                            ? (double)expected_keys * std::min(0.5, 0.04 * lam / 1.5 * lam / 1.5 + 0.01)
                            : (double)expected_keys * overflow_fraction((double)expected_keys / (double)nb);
    p->stashBuckets = next_pow2(std::max<uint64_t>(1u << 12, (uint64_t)(over * 0.75) + 1));
    g.stashBuckets = p->stashBuckets;
    IBS_CUDA(cudaMalloc(&p->buckets, nb * 32), "panel table alloc");
    IBS_CUDA(cudaMemset(p->buckets, 0, nb * 32), "panel table init");
    IBS_CUDA(cudaMalloc(&p->stash, p->stashBuckets * 32), "panel stash alloc");
    k_stash_init<<<grid_for(p->stashBuckets * 2), 256>>>(p->stash, p->stashBuckets * 2);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "panel stash init");
    IBS_CUDA(cudaMalloc(&p->dErr, sizeof(int)), "panel alloc");
    IBS_CUDA(cudaMemset(p->dErr, 0, sizeof(int)), "panel alloc");
    IBS_CUDA(cudaMalloc(&p->dCounters, 32), "panel alloc");
    p->deviceBytes = nb * 32 + p->stashBuckets * 32;
    *out = p.release();
    return IBS_OK;
}

// Doubles the stash and moves its entries over.
static ibs_status grow_stash(ibs_panel_table *p)
{
    const uint64_t nb = p->stashBuckets * 2;
    ulonglong2 *fresh = nullptr;
    IBS_CUDA(cudaMalloc(&fresh, nb * 32), "panel stash growth");
    std::unique_ptr<ulonglong2, cudaError_t (*)(void *)> guard(fresh, cudaFree);
    k_stash_init<<<grid_for(nb * 2), 256>>>(fresh, nb * 2);
    IBS_LAUNCHED();
    IBS_CUDA(cudaMemset(p->dErr, 0, sizeof(int)), "panel stash growth");
    k_stash_move<<<grid_for(p->stashBuckets * 2), 256>>>(p->stash, p->stashBuckets * 2,
                                                         reinterpret_cast<unsigned long long *>(fresh), nb,
                                                         p->dErr);
    IBS_LAUNCHED();
    int err = 0;
    IBS_CUDA(cudaMemcpy(&err, p->dErr, sizeof(int), cudaMemcpyDeviceToHost), "panel stash growth");
    if (err) { // cannot happen: the new stash has twice the entries
        set_error("panel table: stash growth lost entries");
        return IBS_ERR_STATE;
    }
    cudaFree(p->stash);
    p->stash = guard.release();
    p->deviceBytes += p->stashBuckets * 32;
    p->stashBuckets = nb;
    p->geom.stashBuckets = nb;
    p->stashGrowths++;
    return IBS_OK;
}

// A panel whose table was handed to a server keeps only its handle.
static ibs_status check_live(const ibs_panel_table *p)
{
    if (p->buckets)
        return IBS_OK;
    set_error("panel table: its device table was released to a server");
    return IBS_ERR_STATE;
}

static ibs_status panel_add_device_codes(ibs_panel_table *p, const uint64_t *dCodes, uint64_t n)
{
    if (check_live(p) != IBS_OK)
        return IBS_ERR_STATE;
    if (p->nSamples >= kMaxSamples) {
        set_error("panel table already holds " + std::to_string(kMaxSamples) + " samples");
        return IBS_ERR_CAPACITY;
    }
    const auto t0 = std::chrono::steady_clock::now();
    const uint32_t bit = p->nSamples;
    if (p->graph) { // the captured scan holds the old sample count
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    // keys go in chunks, so the build's scratch stays small next to the table
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(n, kBuildChunk));
    uint64_t *pending = nullptr, *failed = nullptr;
    IBS_CUDA(cudaMalloc(&pending, chunk * 8), "panel pending alloc");
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> g1(pending, cudaFree);
    IBS_CUDA(cudaMalloc(&failed, chunk * 8), "panel pending alloc");
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> g2(failed, cudaFree);
    unsigned long long *cnt = p->dCounters; // [0] pending, [2] failed
    for (uint64_t c0 = 0; c0 < n; c0 += chunk) {
        const uint64_t m = std::min<uint64_t>(chunk, n - c0);
        IBS_CUDA(cudaMemset(cnt, 0, 8), "panel build");
        View v = p->view();
        k_find<<<grid_for(m), 256>>>(v, reinterpret_cast<uint32_t *>(p->buckets),
                                     reinterpret_cast<unsigned long long *>(p->stash), dCodes + c0, m, bit,
                                     pending, cnt);
        IBS_LAUNCHED();
        unsigned long long nPend = 0;
        IBS_CUDA(cudaMemcpy(&nPend, cnt, 8, cudaMemcpyDeviceToHost), "panel build find");
        const uint64_t *todo = pending;
        for (int round = 0; nPend; ++round) {
            if (round > 40) { // each round doubles the stash: 2^40 x its start is out of reach
                set_error("panel table: stash growth did not converge");
                return IBS_ERR_STATE;
            }
            IBS_CUDA(cudaMemset(cnt + 2, 0, 8), "panel build");
            View w = p->view();
            k_insert<<<grid_for(nPend), 256>>>(w, reinterpret_cast<uint32_t *>(p->buckets),
                                               reinterpret_cast<unsigned long long *>(p->stash), todo, nPend,
                                               bit, todo == failed ? pending : failed, cnt + 2);
            IBS_LAUNCHED();
            unsigned long long nFail = 0;
            IBS_CUDA(cudaMemcpy(&nFail, cnt + 2, 8, cudaMemcpyDeviceToHost), "panel build insert");
            if (!nFail)
                break;
            ibs_status st = grow_stash(p);
            if (st != IBS_OK)
                return st;
            todo = todo == failed ? pending : failed;
            nPend = nFail;
        }
    }
    p->nSamples++;
    p->keysAdded += n;
    p->buildSeconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return IBS_OK;
}

extern "C" ibs_status ibs_panel_table_add_codes(ibs_panel_table *p, const uint64_t *codes, uint64_t n,
                                                int codes_on_device)
{
    clear_error();
    if (!p || (n && !codes)) {
        set_error("ibs_panel_table_add_codes: bad argument");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(p->device);
    if (codes_on_device)
        return panel_add_device_codes(p, codes, n);
    uint64_t *d = nullptr;
    IBS_CUDA(cudaMalloc(&d, std::max<uint64_t>(n, 1) * 8), "codes alloc");
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> guard2(d, cudaFree);
    IBS_CUDA(cudaMemcpy(d, codes, n * 8, cudaMemcpyHostToDevice), "codes upload");
    return panel_add_device_codes(p, d, n);
}

extern "C" ibs_status ibs_panel_table_add_kmc(ibs_panel_table *p, const char *prefix)
{
    clear_error();
    if (!p || !prefix) {
        set_error("ibs_panel_table_add_kmc: bad argument");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(p->device);
    uint64_t *d = nullptr, n = 0;
    uint32_t k = 0;
    ibs_status s = decode_kmc(prefix, p->device, &d, &n, &k);
    if (s != IBS_OK)
        return s;
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> guard2(d, cudaFree);
    if (k != p->geom.k) {
        set_error(std::string("panel table: ") + prefix + " has k=" + std::to_string(k) +
                  " but the panel has k=" + std::to_string(p->geom.k) + "; a panel shares one k");
        return IBS_ERR_ARG;
    }
    return panel_add_device_codes(p, d, n);
}

extern "C" ibs_status ibs_panel_table_info_get(const ibs_panel_table *p, ibs_table_info *info,
                                               uint32_t *n_samples)
{
    clear_error();
    if (!p || !info) {
        set_error("ibs_panel_table_info_get: bad argument");
        return IBS_ERR_ARG;
    }
    memset(info, 0, sizeof *info);
    info->k = p->geom.k;
    info->format = p->geom.format;
    info->fp_bits = p->geom.fpBits;
    info->n_keys = p->keysAdded;
    info->n_buckets = p->geom.nBuckets;
    info->stash_buckets = p->stashBuckets;
    info->device_bytes = p->deviceBytes;
    info->build_seconds = p->buildSeconds;
    if (n_samples)
        *n_samples = p->nSamples;
    return IBS_OK;
}

extern "C" ibs_status ibs_panel_table_probe(ibs_panel_table *p, const uint64_t *codes, uint64_t n,
                                            uint32_t *masks)
{
    clear_error();
    if (!p || (n && (!codes || !masks))) {
        set_error("ibs_panel_table_probe: bad argument");
        return IBS_ERR_ARG;
    }
    if (check_live(p) != IBS_OK)
        return IBS_ERR_STATE;
    if (!n)
        return IBS_OK;
    DeviceGuard guard(p->device);
    uint64_t *dc = nullptr;
    uint32_t *dm = nullptr;
    IBS_CUDA(cudaMalloc(&dc, n * 8), "probe alloc");
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> g1(dc, cudaFree);
    IBS_CUDA(cudaMalloc(&dm, n * 4), "probe alloc");
    std::unique_ptr<uint32_t, cudaError_t (*)(void *)> g2(dm, cudaFree);
    IBS_CUDA(cudaMemcpy(dc, codes, n * 8, cudaMemcpyHostToDevice), "probe upload");
    k_probe_masks<<<grid_for(n), 256>>>(p->view(), dc, n, dm);
    IBS_LAUNCHED();
    IBS_CUDA(cudaMemcpy(masks, dm, n * 4, cudaMemcpyDeviceToHost), "probe download");
    return IBS_OK;
}

// Bucket-range passes of a scan: one while the bucket array is within the
// pass size (ibs_tuning.panel_pass_mb, default 48 GiB), else one per pass
// size of buckets.
static uint32_t pass_count(const ibs_panel_table *p)
{
    const uint64_t passBytes = (tuning().panel_pass_mb ? (uint64_t)tuning().panel_pass_mb : 48ull << 10) << 20;
    const uint64_t bytes = p->geom.nBuckets * 32;
    return (uint32_t)std::max<uint64_t>(1, (bytes + passBytes - 1) / passBytes);
}

// Plan and scratch of (reference, W) for the panel scan.
static ibs_status panel_plan(ibs_panel_table *p, const ibs_reference *ref, uint32_t W)
{
    const uint32_t spanLen = tuning().panel_span_len;
    if (p->planRef == ref && p->plan.W == W && p->plan.dWin && p->planLens == ref->lens &&
        p->plan.spanLen == spanLen && (pass_count(p) <= 1 || p->dMasks))
        return IBS_OK;
    p->plan.release();
    plan_windows(p->plan, ref->lens, ref->baseOff, W, p->geom.k, spanLen);
    IBS_CUDA(cudaMalloc(&p->plan.dWin, std::max<uint64_t>(p->plan.nWin, 1) * sizeof(WinDesc)), "plan alloc");
    IBS_CUDA(cudaMalloc(&p->plan.dSpan0, (p->plan.nWin + 1) * sizeof(uint32_t)), "plan alloc");
    if (p->plan.nWin)
        IBS_CUDA(cudaMemcpy(p->plan.dWin, p->plan.win.data(), p->plan.nWin * sizeof(WinDesc),
                            cudaMemcpyHostToDevice),
                 "plan upload");
    IBS_CUDA(cudaMemcpy(p->plan.dSpan0, p->plan.span0.data(), (p->plan.nWin + 1) * sizeof(uint32_t),
                        cudaMemcpyHostToDevice),
             "plan upload");
    const uint64_t need = std::max<uint64_t>(1, p->plan.nSpans * kMaxSamples);
    if (p->spansCap < need) {
        cudaFree(p->dSpans);
        p->dSpans = nullptr;
        p->spansCap = 0;
        IBS_CUDA(cudaMalloc(&p->dSpans, need * sizeof(SegStats)), "panel span scratch");
        p->spansCap = need;
    }
    // per-position sample masks between the passes of a multi-pass scan
    cudaFree(p->dMasks);
    p->dMasks = nullptr;
    if (pass_count(p) > 1)
        IBS_CUDA(cudaMalloc(&p->dMasks, std::max<uint64_t>(1, p->plan.nSpans * p->plan.spanLen) * 2),
                 "panel mask scratch");
    p->planRef = ref;
    p->planLens = ref->lens;
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    return IBS_OK;
}

// The span kernel's launches of one scan: one launch, or one per
// bucket-range pass and a statistics launch.
template <int NB, bool PM>
static ibs_status enqueue_spans(ibs_panel_table *p, const ibs_reference *ref, uint32_t passes, int grid,
                                cudaStream_t st)
{
    const ScanPlan &pl = p->plan;
    if (passes <= 1) {
        IBS_CUDA(cudaMemsetAsync(p->dCounters + 1, 0, 8, st), "panel work reset");
        k_panel_spans<NB, kScan, PM><<<grid, 256, 0, st>>>(p->view(), ref->dSeq, ref->dMask, pl.dWin, pl.dSpan0,
                                                       (uint32_t)pl.nWin, pl.nSpans, pl.spanLen, p->nSamples,
                                                       p->dCounters + 1, p->dSpans, nullptr, 0, 0, false);
        IBS_LAUNCHED();
        return IBS_OK;
    }
    const uint64_t nb = p->geom.nBuckets;
    for (uint32_t i = 0; i < passes; ++i) {
        IBS_CUDA(cudaMemsetAsync(p->dCounters + 1, 0, 8, st), "panel work reset");
        k_panel_spans<NB, kMaskPass, PM><<<grid, 256, 0, st>>>(
            p->view(), ref->dSeq, ref->dMask, pl.dWin, pl.dSpan0, (uint32_t)pl.nWin, pl.nSpans, pl.spanLen,
            p->nSamples, p->dCounters + 1, p->dSpans, p->dMasks, nb * i / passes, nb * (i + 1) / passes, i == 0);
        IBS_LAUNCHED();
    }
    IBS_CUDA(cudaMemsetAsync(p->dCounters + 1, 0, 8, st), "panel work reset");
    k_panel_spans<NB, kStats, PM><<<grid, 256, 0, st>>>(p->view(), ref->dSeq, ref->dMask, pl.dWin, pl.dSpan0,
                                                    (uint32_t)pl.nWin, pl.nSpans, pl.spanLen, p->nSamples,
                                                    p->dCounters + 1, p->dSpans, p->dMasks, 0, 0, false);
    IBS_LAUNCHED();
    return IBS_OK;
}

static ibs_status panel_enqueue(ibs_panel_table *p, const ibs_reference *ref, ibs_window *rowsDev,
                                cudaStream_t st)
{
    const ScanPlan &pl = p->plan;
    const uint32_t passes = pass_count(p);
    if (pl.nSpans) {
        const ibs_tuning tu = tuning();
        const int grid = sm_count() * (int)tu.panel_ctas_per_sm;
        const bool pm = p->geom.format == FMT_PANEL_MZ;
        const ibs_status s = tu.panel_blocks_in_flight == 2
                                 ? (pm ? enqueue_spans<2, true>(p, ref, passes, grid, st)
                                       : enqueue_spans<2, false>(p, ref, passes, grid, st))
                                 : (pm ? enqueue_spans<4, true>(p, ref, passes, grid, st)
                                       : enqueue_spans<4, false>(p, ref, passes, grid, st));
        if (s != IBS_OK)
            return s;
    }
    if (pl.nWin && p->nSamples) {
        k_panel_finalize<<<grid_for(pl.nWin * p->nSamples), 256, 0, st>>>(
            pl.dWin, pl.dSpan0, pl.nWin, pl.nSpans, p->nSamples, p->dSpans, (int)p->geom.k, rowsDev);
        IBS_LAUNCHED();
    }
    IBS_CUDA(cudaGetLastError(), "panel scan launch");
    return IBS_OK;
}

extern "C" ibs_status ibs_panel_table_scan_async(ibs_panel_table *p, ibs_reference *ref, uint32_t W,
                                                 ibs_window *rows_dev, uint64_t cap, void *stream)
{
    clear_error();
    if (!p || !ref || p->device != ref->device) {
        set_error("ibs_panel_table_scan_async: bad argument");
        return IBS_ERR_ARG;
    }
    if (W <= p->geom.k) {
        set_error("window size " + std::to_string(W) + " must be larger than k (" +
                  std::to_string(p->geom.k) + ")");
        return IBS_ERR_ARG;
    }
    const uint64_t nWin = ibs_window_count(ref->lens.data(), (uint32_t)ref->lens.size(), W, p->geom.k);
    if (nWin * p->nSamples > cap || (nWin && p->nSamples && !rows_dev)) {
        set_error("ibs_panel_table_scan_async: row capacity too small (samples x windows)");
        return IBS_ERR_ARG;
    }
    if (check_live(p) != IBS_OK)
        return IBS_ERR_STATE;
    DeviceGuard guard(p->device);
    ibs_status s = panel_plan(p, ref, W);
    if (s != IBS_OK)
        return s;
    cudaStream_t st = (cudaStream_t)stream;
    // Replay the captured scan when (reference, W, rows, stream) repeat:
    // the work reset, the span kernel and the finalizer as one graph.
    const void *key[3] = {ref, rows_dev, stream};
    const ibs_tuning tu = tuning();
    const uint32_t shape[3] = {tu.panel_ctas_per_sm, tu.panel_blocks_in_flight, pass_count(p)};
    if (p->graph && p->graphW == W && !memcmp(key, p->graphKey, sizeof key) &&
        !memcmp(shape, p->graphShape, sizeof shape)) {
        IBS_CUDA(cudaGraphLaunch(p->graph, st), "panel graph launch");
        IBS_LAUNCHED();
        return IBS_OK;
    }
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    cudaStream_t cap_st = nullptr;
    IBS_CUDA(cudaStreamCreateWithFlags(&cap_st, cudaStreamNonBlocking), "capture stream");
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(cap_st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        s = panel_enqueue(p, ref, rows_dev, cap_st);
        e = cudaStreamEndCapture(cap_st, &g);
    }
    if (e == cudaSuccess && s == IBS_OK)
        e = cudaGraphInstantiate(&p->graph, g, 0);
    if (g)
        cudaGraphDestroy(g);
    cudaStreamDestroy(cap_st);
    if (s != IBS_OK)
        return s;
    IBS_CUDA(e, "panel graph capture");
    memcpy(p->graphKey, key, sizeof key);
    memcpy(p->graphShape, shape, sizeof shape);
    p->graphW = W;
    IBS_CUDA(cudaGraphLaunch(p->graph, st), "panel graph launch");
    return IBS_OK;
}

extern "C" ibs_status ibs_panel_table_scan(ibs_panel_table *p, ibs_reference *ref, uint32_t W,
                                           ibs_window *rows, uint64_t cap)
{
    clear_error();
    if (!p || !ref) {
        set_error("ibs_panel_table_scan: bad argument");
        return IBS_ERR_ARG;
    }
    const uint64_t nWin = ibs_window_count(ref->lens.data(), (uint32_t)ref->lens.size(), W, p->geom.k);
    const uint64_t need = nWin * p->nSamples;
    if (need > cap || (need && !rows)) {
        set_error("ibs_panel_table_scan: row capacity too small (samples x windows)");
        return IBS_ERR_ARG;
    }
    if (check_live(p) != IBS_OK)
        return IBS_ERR_STATE;
    DeviceGuard guard(p->device);
    ibs_window *d = nullptr;
    IBS_CUDA(cudaMalloc(&d, std::max<uint64_t>(need, 1) * sizeof(ibs_window)), "row alloc");
    std::unique_ptr<ibs_window, cudaError_t (*)(void *)> g(d, cudaFree);
    cudaStream_t st = nullptr;
    IBS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream create");
    ibs_status s = ibs_panel_table_scan_async(p, ref, W, d, need, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if (s == IBS_OK && e == cudaSuccess && need)
        e = cudaMemcpy(rows, d, need * sizeof(ibs_window), cudaMemcpyDeviceToHost);
    // the graph was captured for this call's temporary buffers: drop it
    if (p->graph && p->graphKey[1] == d) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    cudaStreamDestroy(st);
    if (s != IBS_OK)
        return s;
    IBS_CUDA(e, "panel scan");
    return IBS_OK;
}

namespace ibs {
// Frees the panel's device table (the server keeps a host image of it).
void panel_release_table(ibs_panel_table *p)
{
    DeviceGuard guard(p->device);
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    cudaFree(p->buckets);
    cudaFree(p->stash);
    p->buckets = nullptr;
    p->stash = nullptr;
    p->deviceBytes = 0;
}
} // namespace ibs

extern "C" void ibs_panel_table_close(ibs_panel_table *p)
{
    if (!p)
        return;
    {
        DeviceGuard guard(p->device);
        if (p->graph)
            cudaGraphExecDestroy(p->graph);
        p->plan.release();
        cudaFree(p->dSpans);
        cudaFree(p->dMasks);
        cudaFree(p->buckets);
        cudaFree(p->stash);
        cudaFree(p->dErr);
        cudaFree(p->dCounters);
    }
    delete p;
}
