// The window scan on sm_100a.
//
// Work unit: a span = up to spanLen consecutive k-mer positions of ONE
// window (windows never share a span). One warp owns a span: lane i takes
// position p+i of each 32-position block, encodes its k-mer straight from the
// 2-bit reference (two 64-bit words, a funnel shift, a bit reversal for the
// forward strand and a complement for the reverse strand), probes the table
// with one 32-byte bucket load, and the warp folds the block's hit/valid
// ballots into the span's statistics with popc and warp reductions. A second
// kernel folds each window's span summaries in order into its row.
//
// This restates, as one fused device pass, the reference's per-window loop:
// KmerCodec::getCanonicalCodes (src/KmerCodec.hpp:38-61), the probe
// (src/gpu/ProbeCore.hpp:113-129), BitStats::run
// (src/gpu/EncodeProbeCore.hpp:338-370) and Window::addVariationOriginal
// (src/Window.hpp:29-36), with the windows of chunkSequences
// (src/Utils.hpp:296-327).
#include "ibs_internal.cuh"
#include "mz_scan.cuh"
#include "scan_device.cuh"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>

namespace ibs {

constexpr uint32_t FULL = 0xffffffffu;

static std::mutex g_tuneMu;
// Defaults: the autotuner's best point on the B200 (gpu-ibs_b200/tuning/b200.json,
// plain 2 Gbp x 2.19e9 k-mers): minimizer table at 1.5 keys per 32-byte
// sector, spans of 2048 positions, 2 blocks in flight, 512 threads, 16 CTAs
// per SM.
// Joint-table scans (the autotuner's best point on the 16-sample panel at
// half size): spans of 8192 positions, 4 CTAs of 256 threads per SM, 2
// blocks in flight, 3 keys per 5-slot bucket.
static ibs_tuning g_tune = {2048, 2, 512, 16, 1.5, FMT_MZ8, 0, 8192, 4, 3.0, 2, {0, 0, 0}};

const ibs_tuning &tuning() { return g_tune; }

using dev::canonical_at;

// Feeds NB consecutive 32-position blocks' ballots to the span fold.
template <int NB>
__device__ __forceinline__ void fold_blocks(dev::LaneFold &fold, const uint32_t (&V)[NB], const uint32_t (&H)[NB],
                                            uint32_t lane, int k)
{
#pragma unroll
    for (int b = 0; b < NB; ++b)
        fold.push(V[b], H[b], lane, k);
}

__device__ __forceinline__ uint32_t window_of_span(const uint32_t *__restrict__ span0,
                                                   uint32_t nWin, uint64_t s)
{
    uint32_t lo = 0, hi = nWin - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(span0 + mid) <= s)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <uint32_t FMT, int NB>
__global__ void __launch_bounds__(512) k_scan_spans(TableView t, const uint64_t *__restrict__ seq,
                                                    const uint64_t *__restrict__ mask,
                                                    const WinDesc *__restrict__ win,
                                                    const uint32_t *__restrict__ span0,
                                                    uint32_t nWin, uint64_t s0, uint64_t s1,
                                                    uint32_t spanLen, SegStats *__restrict__ out)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = t.g.k;
    const uint64_t kmask = key_mask(2 * k);
    const uint64_t kbits = (1ull << k) - 1; // k <= 32
    for (uint64_t s = s0 + warp; s < s1; s += nWarps) {
        const uint32_t w = window_of_span(span0, nWin, s);
        const uint64_t base = win[w].base;
        const uint32_t nPos = win[w].nPos;
        const uint32_t p0 = (uint32_t)(s - __ldg(span0 + w)) * spanLen;
        const uint32_t p1 = min(p0 + spanLen, nPos);
        dev::LaneFold fold;
        for (uint32_t p = p0; p < p1; p += 32 * NB) {
            uint4 v0[NB], v1[NB];
            uint64_t code[NB], fp[NB];
            bool valid[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const uint32_t q = p + 32 * b + lane;
                const bool inSpan = q < p1;
                // lanes past the span read a position inside it (no access
                // beyond the contig's padded words) and are masked out
                const uint64_t G = base + (inSpan ? q : p0);
                bool acgt;
                code[b] = canonical_at(seq, mask, G, k, kmask, kbits, acgt);
                valid[b] = inSpan && acgt;
                const uint64_t h = perm_hash(code[b], t.g.bits);
                const uint64_t r = bucket_of(h, t.g);
                fp[b] = fp_of(h, t.g);
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
                    const uint32_t m = bucket_match<FMT>(v0[b], v1[b], fp[b]);
                    hit = m == 1u || (m == 2u && stash_lookup(t, code[b]));
                }
                V[b] = __ballot_sync(FULL, valid[b]);
                H[b] = __ballot_sync(FULL, hit);
            }
            fold_blocks<NB>(fold, V, H, lane, (int)k);
        }
        const SegStats acc = fold.finish((int)k);
        if (lane == 0)
            out[s] = acc;
    }
}

// The scan over a wide-key table (33 <= k <= 64, format FMT_WIDE): the span
// loop of k_scan_spans with each lane's k-mer read as a 128-bit canonical
// code from three packed words and the warp's 32 codes looked up together,
// 8 lanes reading each 128-byte line (wide::lookup_warp).
// Restates the reference's string path for these k: canonical k-mer strings
// of the window (getCanonicalKmersLegacy, src/Utils.hpp:102-125: toupper,
// k-mers with a non-ACGT byte skipped, the smaller of the k-mer and its
// reverse complement) each looked up in the database
// (getStatsFromSequenceLegacy, src/KmerDatabase.hpp:675-708), with the same
// statistics fold.
__global__ void __launch_bounds__(256) k_scan_spans_wide(wide::View t, const uint64_t *__restrict__ seq,
                                                         const uint64_t *__restrict__ mask,
                                                         const WinDesc *__restrict__ win,
                                                         const uint32_t *__restrict__ span0, uint32_t nWin,
                                                         uint64_t s0, uint64_t s1, uint32_t spanLen,
                                                         SegStats *__restrict__ out)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = t.k;
    for (uint64_t s = s0 + warp; s < s1; s += nWarps) {
        const uint32_t w = window_of_span(span0, nWin, s);
        const uint64_t base = win[w].base;
        const uint32_t nPos = win[w].nPos;
        const uint32_t p0 = (uint32_t)(s - __ldg(span0 + w)) * spanLen;
        const uint32_t p1 = min(p0 + spanLen, nPos);
        dev::LaneFold fold;
        for (uint32_t p = p0; p < p1; p += 32) {
            const uint32_t q = p + lane;
            const bool inSpan = q < p1;
            // lanes past the span read a position inside it and are masked out
            const uint64_t G = base + (inSpan ? q : p0);
            bool acgt;
            uint64_t lo, hi;
            wide::canonical_at(seq, mask, G, k, acgt, lo, hi);
            const bool valid = inSpan && acgt;
            const bool hit = wide::lookup_warp(t, lo, hi, valid, lane);
            fold.push(__ballot_sync(FULL, valid), __ballot_sync(FULL, hit), lane, (int)k);
        }
        const SegStats acc = fold.finish((int)k);
        if (lane == 0)
            out[s] = acc;
    }
}

// The scan over a minimizer-line table (formats MZ8 and MZ6): one warp per
// span, the span's statistics from mz_span_stats (mz_scan.cuh). K > 0 fixes
// k at compile time (the shifts and masks fold); K = 0 reads it from the
// table. SEC is the sector layout: FMT_B8X32 (format MZ8) or FMT_B6X40
// (format MZ6).
template <int NB, uint32_t K, uint32_t SEC>
__global__ void __launch_bounds__(512) k_scan_spans_mz(TableView t, const uint64_t *__restrict__ seq,
                                                       const uint64_t *__restrict__ mask,
                                                       const WinDesc *__restrict__ win,
                                                       const uint32_t *__restrict__ span0,
                                                       uint32_t nWin, uint64_t s0, uint64_t s1,
                                                       uint32_t spanLen, SegStats *__restrict__ out)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = K ? K : t.g.k;
    const uint32_t w = mz::w_of(k);
    for (uint64_t s = s0 + warp; s < s1; s += nWarps) {
        const uint32_t wIdx = window_of_span(span0, nWin, s);
        const uint64_t base = win[wIdx].base;
        const uint32_t nPos = win[wIdx].nPos;
        const uint32_t p0 = (uint32_t)(s - __ldg(span0 + wIdx)) * spanLen;
        const uint32_t p1 = min(p0 + spanLen, nPos);
        // last position read: the last m-mer start the window's k-mers use
        const SegStats acc = dev::mz_span_stats<NB, K, SEC>(t, seq, mask, base, p0, p1, nPos - 1 + (w - 1), lane);
        if (lane == 0)
            out[s] = acc;
    }
}

__global__ void k_finalize(const WinDesc *__restrict__ win, const uint32_t *__restrict__ span0,
                           uint64_t nWin, const SegStats *__restrict__ spans, int k,
                           ibs_window *__restrict__ rows)
{
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nWin;
         w += (uint64_t)gridDim.x * blockDim.x) {
        SegStats acc = seg_empty();
        for (uint32_t s = span0[w]; s < span0[w + 1]; ++s)
            acc = seg_combine(acc, spans[s], k);
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
        rows[w] = o;
    }
}

static int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

void ScanPlan::release()
{
    cudaFree(dWin);
    cudaFree(dSpan0);
    cudaFree(dSpans);
    dWin = nullptr;
    dSpan0 = nullptr;
    dSpans = nullptr;
    W = k = spanLen = 0;
    nWin = nSpans = 0;
    win.clear();
    span0.clear();
}

void plan_windows(ScanPlan &p, const std::vector<uint64_t> &lens,
                  const std::vector<uint64_t> &baseOff, uint32_t W, uint32_t k, uint32_t spanLen)
{
    p.win.clear();
    p.span0.clear();
    p.W = W;
    p.k = k;
    p.spanLen = spanLen;
    uint64_t spans = 0;
    const uint64_t step = (uint64_t)W - k;
    for (size_t c = 0; c < lens.size(); ++c) {
        const uint64_t len = lens[c];
        for (uint64_t j = 0; j < len; j += step) {
            const uint64_t end = std::min<uint64_t>(j + W, len);
            const uint64_t nb = end - j;
            WinDesc d;
            d.base = baseOff[c] + j;
            d.nPos = nb >= k ? (uint32_t)(nb - k + 1) : 0u;
            d.start = (int32_t)j;
            d.end = (int32_t)end;
            d.pad = 0;
            p.win.push_back(d);
            p.span0.push_back((uint32_t)spans);
            spans += (d.nPos + spanLen - 1) / spanLen;
        }
    }
    p.span0.push_back((uint32_t)spans);
    p.nWin = p.win.size();
    p.nSpans = spans;
}

template <uint32_t FMT, int NB>
static void launch_nb(const ibs_table *t, const uint64_t *dSeq, const uint64_t *dMask, const ScanPlan &p,
                      uint64_t s0, uint64_t s1, SegStats *dSpans, cudaStream_t st, int grid, int threads)
{
    if (FMT == FMT_MZ8 && t->geom.k == 25)
        k_scan_spans_mz<NB, 25, FMT_B8X32><<<grid, threads, 0, st>>>(t->view(), dSeq, dMask, p.dWin, p.dSpan0,
                                                                     (uint32_t)p.nWin, s0, s1, p.spanLen, dSpans);
    else if (FMT == FMT_MZ8)
        k_scan_spans_mz<NB, 0, FMT_B8X32><<<grid, threads, 0, st>>>(t->view(), dSeq, dMask, p.dWin, p.dSpan0,
                                                                    (uint32_t)p.nWin, s0, s1, p.spanLen, dSpans);
    else if (FMT == FMT_MZ6 && t->geom.k == 31)
        k_scan_spans_mz<NB, 31, FMT_B6X40><<<grid, threads, 0, st>>>(t->view(), dSeq, dMask, p.dWin, p.dSpan0,
                                                                     (uint32_t)p.nWin, s0, s1, p.spanLen, dSpans);
    else if (FMT == FMT_MZ6)
        k_scan_spans_mz<NB, 0, FMT_B6X40><<<grid, threads, 0, st>>>(t->view(), dSeq, dMask, p.dWin, p.dSpan0,
                                                                    (uint32_t)p.nWin, s0, s1, p.spanLen, dSpans);
    else
        k_scan_spans<FMT, NB><<<grid, threads, 0, st>>>(t->view(), dSeq, dMask, p.dWin, p.dSpan0,
                                                        (uint32_t)p.nWin, s0, s1, p.spanLen, dSpans);
}

template <uint32_t FMT>
static void launch_spans_fmt(const ibs_table *t, const uint64_t *dSeq, const uint64_t *dMask,
                             const ScanPlan &p, uint64_t s0, uint64_t s1, SegStats *dSpans,
                             cudaStream_t st)
{
    const ibs_tuning tu = tuning();
    const int threads = (int)tu.block_threads;
    const uint64_t warpsPerCta = threads / 32;
    const uint64_t want = (s1 - s0 + warpsPerCta - 1) / warpsPerCta;
    const uint64_t cap = (uint64_t)sm_count() * tu.ctas_per_sm;
    const int grid = (int)std::max<uint64_t>(1, std::min(want, cap));
    switch (tu.blocks_in_flight) {
    case 1: launch_nb<FMT, 1>(t, dSeq, dMask, p, s0, s1, dSpans, st, grid, threads); break;
    case 2: launch_nb<FMT, 2>(t, dSeq, dMask, p, s0, s1, dSpans, st, grid, threads); break;
    case 8: launch_nb<FMT, 8>(t, dSeq, dMask, p, s0, s1, dSpans, st, grid, threads); break;
    default: launch_nb<FMT, 4>(t, dSeq, dMask, p, s0, s1, dSpans, st, grid, threads); break;
    }
}

// The wide-key scan: 256 threads, as many CTAs as are resident at once.
static void launch_spans_wide(const ibs_table *t, const uint64_t *dSeq, const uint64_t *dMask, const ScanPlan &p,
                              uint64_t s0, uint64_t s1, SegStats *dSpans, cudaStream_t st)
{
    const int threads = 256;
    int perSm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_scan_spans_wide, threads, 0) != cudaSuccess ||
        perSm < 1)
        perSm = 1;
    const uint64_t want = (s1 - s0 + 7) / 8;
    const uint64_t cap = (uint64_t)sm_count() * perSm;
    const int grid = (int)std::max<uint64_t>(1, std::min(want, cap));
    k_scan_spans_wide<<<grid, threads, 0, st>>>(t->wide, dSeq, dMask, p.dWin, p.dSpan0, (uint32_t)p.nWin, s0, s1,
                                                p.spanLen, dSpans);
}

static ibs_status launch_spans(const ibs_table *t, const uint64_t *dSeq, const uint64_t *dMask,
                               const ScanPlan &p, uint64_t s0, uint64_t s1, SegStats *dSpans,
                               cudaStream_t st)
{
    if (s1 <= s0)
        return IBS_OK;
    if (t->geom.format == FMT_WIDE)
        launch_spans_wide(t, dSeq, dMask, p, s0, s1, dSpans, st);
    else if (t->geom.format == FMT_B8X32)
        launch_spans_fmt<FMT_B8X32>(t, dSeq, dMask, p, s0, s1, dSpans, st);
    else if (t->geom.format == FMT_MZ8)
        launch_spans_fmt<FMT_MZ8>(t, dSeq, dMask, p, s0, s1, dSpans, st);
    else if (t->geom.format == FMT_MZ6)
        launch_spans_fmt<FMT_MZ6>(t, dSeq, dMask, p, s0, s1, dSpans, st);
    else
        launch_spans_fmt<FMT_B6X40>(t, dSeq, dMask, p, s0, s1, dSpans, st);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "scan kernel launch");
    return IBS_OK;
}

ibs_status launch_scan(const ibs_table *t, const uint64_t *dSeq, const uint64_t *dMask,
                       const ScanPlan &p, uint64_t s0, uint64_t s1, cudaStream_t st)
{
    return launch_spans(t, dSeq, dMask, p, s0, s1, p.dSpans, st);
}

static ibs_status launch_finalize_with(const ScanPlan &p, uint32_t k, const SegStats *dSpans,
                                       ibs_window *dRows, cudaStream_t st)
{
    if (!p.nWin)
        return IBS_OK;
    const int threads = 256;
    const uint64_t want = (p.nWin + threads - 1) / threads;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sm_count() * 8));
    k_finalize<<<grid, threads, 0, st>>>(p.dWin, p.dSpan0, p.nWin, dSpans, (int)k, dRows);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "finalize kernel launch");
    return IBS_OK;
}

ibs_status launch_finalize(const ScanPlan &p, uint32_t k, ibs_window *dRows, cudaStream_t st)
{
    return launch_finalize_with(p, k, p.dSpans, dRows, st);
}

ibs_status launch_panel(ibs_table *const *tables, uint32_t nTables, const uint64_t *dSeq,
                        const uint64_t *dMask, const ScanPlan &p, ibs_window *dRows,
                        SegStats *dSpans, cudaStream_t st)
{
    for (uint32_t i = 0; i < nTables; ++i) {
        ibs_status s = launch_spans(tables[i], dSeq, dMask, p, 0, p.nSpans, dSpans, st);
        if (s != IBS_OK)
            return s;
        s = launch_finalize_with(p, p.k, dSpans, dRows + (uint64_t)i * p.nWin, st);
        if (s != IBS_OK)
            return s;
    }
    return IBS_OK;
}

// Uploads a plan's window and span arrays and sizes its span scratch.
static ibs_status upload_plan(ScanPlan &p, cudaStream_t st)
{
    IBS_CUDA(cudaMalloc(&p.dWin, std::max<uint64_t>(p.nWin, 1) * sizeof(WinDesc)), "plan alloc");
    IBS_CUDA(cudaMalloc(&p.dSpan0, (p.nWin + 1) * sizeof(uint32_t)), "plan alloc");
    IBS_CUDA(cudaMalloc(&p.dSpans, std::max<uint64_t>(p.nSpans, 1) * sizeof(SegStats)),
             "span scratch alloc");
    if (p.nWin)
        IBS_CUDA(cudaMemcpyAsync(p.dWin, p.win.data(), p.nWin * sizeof(WinDesc),
                                 cudaMemcpyHostToDevice, st),
                 "plan upload");
    IBS_CUDA(cudaMemcpyAsync(p.dSpan0, p.span0.data(), (p.nWin + 1) * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, st),
             "plan upload");
    return IBS_OK;
}

// ---------------------------------------------------------------------------
// host packing
// ---------------------------------------------------------------------------
void packed_offsets(const uint64_t *lens, uint32_t n, std::vector<uint64_t> &off, uint64_t &seqWords,
                    uint64_t &maskWords)
{
    off.resize(n);
    uint64_t b = 0;
    for (uint32_t c = 0; c < n; ++c) {
        off[c] = b;
        b += round_up64(lens[c]);
    }
    seqWords = b / 32 + 1;
    maskWords = b / 64 + 1;
}

// The reference's packWindow (src/gpu/EncodeProbeCore.hpp:157-186) over a
// whole contig starting on a mask-word boundary: 64 bases -> 2 seq words and
// 1 mask word per step.
static void pack_contig(const char *s, uint64_t len, uint64_t *seq, uint64_t *mask)
{
    static const struct Tab {
        uint8_t v[256];
        Tab()
        {
            memset(v, 4, sizeof v);
            v[(uint8_t)'A'] = v[(uint8_t)'a'] = 0;
            v[(uint8_t)'C'] = v[(uint8_t)'c'] = 1;
            v[(uint8_t)'G'] = v[(uint8_t)'g'] = 2;
            v[(uint8_t)'T'] = v[(uint8_t)'t'] = 3;
        }
    } tab;
    for (uint64_t b0 = 0; b0 < len; b0 += 64) {
        uint64_t sw0 = 0, sw1 = 0, mw = 0;
        const uint64_t n = std::min<uint64_t>(64, len - b0);
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t c = tab.v[(uint8_t)s[b0 + i]];
            if (c > 3) {
                mw |= 1ull << i;
                c = 0;
            }
            if (i < 32)
                sw0 |= (uint64_t)c << (2 * i);
            else
                sw1 |= (uint64_t)c << (2 * (i - 32));
        }
        seq[b0 / 32] = sw0;
        seq[b0 / 32 + 1] = sw1;
        mask[b0 / 64] = mw;
    }
}

} // namespace ibs

using namespace ibs;

extern "C" void ibs_packed_words(const uint64_t *lens, uint32_t n, uint64_t *seq_words,
                                 uint64_t *mask_words)
{
    std::vector<uint64_t> off;
    uint64_t sw = 1, mw = 1;
    if (lens || n == 0)
        packed_offsets(lens, n, off, sw, mw);
    if (seq_words)
        *seq_words = sw;
    if (mask_words)
        *mask_words = mw;
}

extern "C" ibs_status ibs_pack_ascii(const char *const *seqs, const uint64_t *lens, uint32_t n,
                                     uint64_t *seq2bit, uint64_t *nmask, int threads)
{
    clear_error();
    if ((n && (!seqs || !lens)) || !seq2bit || !nmask) {
        set_error("ibs_pack_ascii: bad argument");
        return IBS_ERR_ARG;
    }
    std::vector<uint64_t> off;
    uint64_t sw, mw;
    packed_offsets(lens, n, off, sw, mw);
    memset(seq2bit, 0, sw * 8);
    memset(nmask, 0, mw * 8);
    // 4 Mbase pieces spread over the threads
    struct Piece {
        uint32_t c;
        uint64_t b0, b1;
    };
    std::vector<Piece> pieces;
    for (uint32_t c = 0; c < n; ++c)
        for (uint64_t b = 0; b < lens[c]; b += (4ull << 20))
            pieces.push_back({c, b, std::min<uint64_t>(lens[c], b + (4ull << 20))});
    if (threads <= 0)
        threads = (int)std::max(1u, std::thread::hardware_concurrency());
    threads = std::max(1, std::min<int>(threads, (int)pieces.size()));
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (size_t i; (i = next.fetch_add(1)) < pieces.size();) {
            const Piece &pc = pieces[i];
            const uint64_t B = off[pc.c] + pc.b0; // multiple of 64
            pack_contig(seqs[pc.c] + pc.b0, pc.b1 - pc.b0, seq2bit + B / 32, nmask + B / 64);
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < threads; ++i)
        pool.emplace_back(work);
    work();
    for (auto &th : pool)
        th.join();
    return IBS_OK;
}

extern "C" uint64_t ibs_window_count(const uint64_t *lens, uint32_t n, uint32_t W, uint32_t k)
{
    if (W <= k || (!lens && n))
        return 0;
    uint64_t tot = 0;
    for (uint32_t c = 0; c < n; ++c)
        tot += windows_in_contig(lens[c], W, k);
    return tot;
}

ibs_status ibs::check_contig_lengths(const uint64_t *lens, uint32_t n, const char *what)
{
    for (uint32_t c = 0; c < n; ++c)
        if (lens[c] > kMaxContigLen) {
            set_error(std::string(what) + ": contig " + std::to_string(c) + " has " + std::to_string(lens[c]) +
                      " bases; window coordinates are 32-bit, so contigs longer than " +
                      std::to_string(kMaxContigLen) + " bases are not supported");
            return IBS_ERR_ARG;
        }
    return IBS_OK;
}

extern "C" ibs_status ibs_window_bounds(const uint64_t *lens, uint32_t n, uint32_t W, uint32_t k,
                                        ibs_window *rows, uint64_t cap)
{
    clear_error();
    if (n && !lens) {
        set_error("ibs_window_bounds: bad argument");
        return IBS_ERR_ARG;
    }
    ibs_status cs = check_contig_lengths(lens, n, "ibs_window_bounds");
    if (cs != IBS_OK)
        return cs;
    if (W <= k) {
        set_error("window size " + std::to_string(W) + " must be larger than k (" +
                  std::to_string(k) + ")");
        return IBS_ERR_ARG;
    }
    const uint64_t need = ibs_window_count(lens, n, W, k);
    if (need > cap || (need && !rows)) {
        set_error("ibs_window_bounds: row capacity too small");
        return IBS_ERR_ARG;
    }
    uint64_t w = 0;
    for (uint32_t c = 0; c < n; ++c)
        for (uint64_t j = 0; j < lens[c]; j += W - k) {
            ibs_window r{};
            r.start = (int32_t)j;
            r.end = (int32_t)std::min<uint64_t>(j + W, lens[c]);
            rows[w++] = r;
        }
    return IBS_OK;
}

static ibs_status reference_new(const uint64_t *lens, uint32_t n, int device, ibs_reference **out,
                                std::unique_ptr<ibs_reference> &r)
{
    if (!out || (n && !lens)) {
        set_error("ibs_reference_create: bad argument");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    ibs_status cs = check_contig_lengths(lens, n, "ibs_reference_create");
    if (cs != IBS_OK)
        return cs;
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd == 0) {
        cudaGetLastError();
        set_error("no usable CUDA device (the scan has no CPU fallback)");
        return IBS_ERR_CUDA;
    }
    if (device < 0 || device >= nd) {
        set_error("device out of range");
        return IBS_ERR_ARG;
    }
    r.reset(new ibs_reference);
    r->device = device;
    r->lens.assign(lens, lens + n);
    packed_offsets(lens, n, r->baseOff, r->seqWords, r->maskWords);
    return IBS_OK;
}

static ibs_status reference_upload(ibs_reference *r, const uint64_t *seq, const uint64_t *mask,
                                   cudaMemcpyKind kind)
{
    IBS_CUDA(cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking), "stream create");
    IBS_CUDA(cudaMalloc(&r->dSeq, r->seqWords * 8), "reference alloc");
    IBS_CUDA(cudaMalloc(&r->dMask, r->maskWords * 8), "reference alloc");
    IBS_CUDA(cudaMemcpy(r->dSeq, seq, r->seqWords * 8, kind), "reference upload");
    IBS_CUDA(cudaMemcpy(r->dMask, mask, r->maskWords * 8, kind), "reference upload");
    return IBS_OK;
}

extern "C" ibs_status ibs_reference_create(const uint64_t *seq2bit, const uint64_t *nmask,
                                           const uint64_t *lens, uint32_t n, int device,
                                           ibs_reference **out)
{
    clear_error();
    std::unique_ptr<ibs_reference> r;
    ibs_status s = reference_new(lens, n, device, out, r);
    if (s != IBS_OK)
        return s;
    if (!seq2bit || !nmask) {
        set_error("ibs_reference_create: bad argument");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(device);
    s = reference_upload(r.get(), seq2bit, nmask, cudaMemcpyHostToDevice);
    if (s != IBS_OK) {
        ibs_reference_free(r.release());
        return s;
    }
    *out = r.release();
    return IBS_OK;
}

ibs_status ibs::reference_adopt(const std::vector<uint64_t> &lens, int device, uint64_t *dSeq, uint64_t *dMask,
                                ibs_reference **out)
{
    std::unique_ptr<ibs_reference> r(new ibs_reference);
    r->device = device;
    r->lens = lens;
    packed_offsets(lens.data(), (uint32_t)lens.size(), r->baseOff, r->seqWords, r->maskWords);
    r->dSeq = dSeq;
    r->dMask = dMask;
    DeviceGuard guard(device);
    const cudaError_t e = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        ibs_reference_free(r.release());
        return cuda_fail(e, "stream create");
    }
    *out = r.release();
    return IBS_OK;
}

extern "C" ibs_status ibs_reference_create_device(const uint64_t *seq2bit, const uint64_t *nmask,
                                                  const uint64_t *lens, uint32_t n, int device,
                                                  ibs_reference **out)
{
    clear_error();
    std::unique_ptr<ibs_reference> r;
    ibs_status s = reference_new(lens, n, device, out, r);
    if (s != IBS_OK)
        return s;
    if (!seq2bit || !nmask) {
        set_error("ibs_reference_create_device: bad argument");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(device);
    s = reference_upload(r.get(), seq2bit, nmask, cudaMemcpyDeviceToDevice);
    if (s != IBS_OK) {
        ibs_reference_free(r.release());
        return s;
    }
    *out = r.release();
    return IBS_OK;
}

extern "C" void ibs_reference_free(ibs_reference *r)
{
    if (!r)
        return;
    {
        DeviceGuard guard(r->device);
        if (r->stream)
            cudaStreamSynchronize(r->stream);
        r->plan.release();
        cudaFree(r->dSeq);
        cudaFree(r->dMask);
        cudaFree(r->dRows);
        cudaFree(r->dPanelSpans);
        if (r->stream)
            cudaStreamDestroy(r->stream);
    }
    delete r;
}

// Makes r->plan describe (W, k); allocates and uploads on a change.
static ibs_status ensure_plan(ibs_reference *r, uint32_t W, uint32_t k)
{
    ScanPlan &p = r->plan;
    const uint32_t spanLen = tuning().span_len;
    if (p.dWin && p.W == W && p.k == k && p.spanLen == spanLen)
        return IBS_OK;
    IBS_CUDA(cudaStreamSynchronize(r->stream), "plan sync");
    p.release();
    plan_windows(p, r->lens, r->baseOff, W, k, spanLen);
    ibs_status s = upload_plan(p, r->stream);
    if (s != IBS_OK)
        p.release();
    return s;
}

static ibs_status check_scan_args(const ibs_table *t, const ibs_reference *ref, uint32_t W,
                                  uint64_t cap, const void *rows)
{
    if (!t || !ref) {
        set_error("scan: null table or reference");
        return IBS_ERR_ARG;
    }
    if (t->device != ref->device) {
        set_error("scan: table and reference live on different devices");
        return IBS_ERR_ARG;
    }
    if (W <= t->geom.k) {
        set_error("window size " + std::to_string(W) + " must be larger than k (" +
                  std::to_string(t->geom.k) + ")");
        return IBS_ERR_ARG;
    }
    const uint64_t need = ibs_window_count(ref->lens.data(), (uint32_t)ref->lens.size(), W,
                                           t->geom.k);
    if (need > cap || (need && !rows)) {
        set_error("scan: row capacity " + std::to_string(cap) + " < " + std::to_string(need) +
                  " windows");
        return IBS_ERR_ARG;
    }
    return IBS_OK;
}

extern "C" ibs_status ibs_scan_async(ibs_table *t, ibs_reference *ref, uint32_t W,
                                     ibs_window *rows_dev, uint64_t cap, void *stream)
{
    clear_error();
    ibs_status s = check_scan_args(t, ref, W, cap, rows_dev);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(t->device);
    s = ensure_plan(ref, W, t->geom.k);
    if (s != IBS_OK)
        return s;
    IBS_CUDA(cudaStreamSynchronize(ref->stream), "plan sync");
    cudaStream_t st = (cudaStream_t)stream;
    s = launch_scan(t, ref->dSeq, ref->dMask, ref->plan, 0, ref->plan.nSpans, st);
    if (s != IBS_OK)
        return s;
    return launch_finalize(ref->plan, t->geom.k, rows_dev, st);
}

extern "C" ibs_status ibs_scan(ibs_table *t, ibs_reference *ref, uint32_t W, ibs_window *rows,
                               uint64_t cap)
{
    clear_error();
    ibs_status s = check_scan_args(t, ref, W, cap, rows);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(t->device);
    s = ensure_plan(ref, W, t->geom.k);
    if (s != IBS_OK)
        return s;
    const uint64_t nWin = ref->plan.nWin;
    if (ref->dRowsCap < nWin) {
        cudaFree(ref->dRows);
        ref->dRows = nullptr;
        ref->dRowsCap = 0;
        IBS_CUDA(cudaMalloc(&ref->dRows, std::max<uint64_t>(nWin, 1) * sizeof(ibs_window)),
                 "row buffer alloc");
        ref->dRowsCap = nWin;
    }
    s = launch_scan(t, ref->dSeq, ref->dMask, ref->plan, 0, ref->plan.nSpans, ref->stream);
    if (s != IBS_OK)
        return s;
    s = launch_finalize(ref->plan, t->geom.k, ref->dRows, ref->stream);
    if (s != IBS_OK)
        return s;
    if (nWin)
        IBS_CUDA(cudaMemcpyAsync(rows, ref->dRows, nWin * sizeof(ibs_window),
                                 cudaMemcpyDeviceToHost, ref->stream),
                 "row download");
    IBS_CUDA(cudaStreamSynchronize(ref->stream), "scan");
    return IBS_OK;
}

extern "C" ibs_status ibs_scan_panel(ibs_table *const *tables, uint32_t n, ibs_reference *ref,
                                     uint32_t W, ibs_window *rows, uint64_t cap)
{
    clear_error();
    if (!tables || n == 0 || !ref) {
        set_error("ibs_scan_panel: bad argument");
        return IBS_ERR_ARG;
    }
    const uint32_t k = tables[0] ? tables[0]->geom.k : 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (!tables[i] || tables[i]->geom.k != k || tables[i]->device != ref->device) {
            set_error("ibs_scan_panel: tables must share k and the reference's device");
            return IBS_ERR_ARG;
        }
    }
    const uint64_t nWin = ibs_window_count(ref->lens.data(), (uint32_t)ref->lens.size(), W, k);
    ibs_status s = check_scan_args(tables[0], ref, W, cap / n, rows);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(ref->device);
    s = ensure_plan(ref, W, k);
    if (s != IBS_OK)
        return s;
    const uint64_t need = nWin * n;
    if (ref->dRowsCap < need) {
        cudaFree(ref->dRows);
        ref->dRows = nullptr;
        ref->dRowsCap = 0;
        IBS_CUDA(cudaMalloc(&ref->dRows, std::max<uint64_t>(need, 1) * sizeof(ibs_window)),
                 "row buffer alloc");
        ref->dRowsCap = need;
    }
    s = launch_panel(tables, n, ref->dSeq, ref->dMask, ref->plan, ref->dRows, ref->plan.dSpans,
                     ref->stream);
    if (s != IBS_OK)
        return s;
    if (need)
        IBS_CUDA(cudaMemcpyAsync(rows, ref->dRows, need * sizeof(ibs_window),
                                 cudaMemcpyDeviceToHost, ref->stream),
                 "row download");
    IBS_CUDA(cudaStreamSynchronize(ref->stream), "panel scan");
    return IBS_OK;
}

// ---------------------------------------------------------------------------
// End-to-end scan over host buffers: the reference is uploaded in window
// groups on a copy stream while earlier groups are scanned on a compute
// stream. Device buffers and pinned staging are kept per device and reused.
// ---------------------------------------------------------------------------
namespace {
struct Workspace {
    int device = -1;
    uint64_t *dSeq = nullptr, *dMask = nullptr;
    uint64_t seqCap = 0, maskCap = 0;
    ibs_window *dRows = nullptr;
    uint64_t rowsCap = 0;
    uint64_t spansCap = 0;
    uint64_t winCap = 0; // windows the plan's device arrays hold
    ScanPlan plan;
    cudaStream_t copy = nullptr, comp = nullptr;
    std::vector<cudaEvent_t> ev;
    uint8_t *stage[2] = {nullptr, nullptr};
    cudaEvent_t stageFree[2] = {nullptr, nullptr};
    uint64_t stageBytes = 0;
};
std::mutex g_wsMu;
Workspace g_ws[16];

ibs_status grow(uint64_t *&p, uint64_t &cap, uint64_t need, const char *what)
{
    if (cap >= need)
        return IBS_OK;
    cudaFree(p);
    p = nullptr;
    cap = 0;
    IBS_CUDA(cudaMalloc(&p, need * 8), what);
    cap = need;
    return IBS_OK;
}

bool is_pinned(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Copies n bytes host -> device on ws.copy, directly when the source is
// pinned, else through the two pinned staging buffers.
ibs_status copy_h2d(Workspace &ws, void *dst, const void *src, uint64_t n, bool pinned)
{
    if (!n)
        return IBS_OK;
    if (pinned) {
        IBS_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, ws.copy), "reference upload");
        return IBS_OK;
    }
    static int slot = 0;
    for (uint64_t o = 0; o < n; o += ws.stageBytes) {
        const uint64_t m = std::min(ws.stageBytes, n - o);
        IBS_CUDA(cudaEventSynchronize(ws.stageFree[slot]), "staging wait");
        memcpy(ws.stage[slot], (const uint8_t *)src + o, m);
        IBS_CUDA(cudaMemcpyAsync((uint8_t *)dst + o, ws.stage[slot], m, cudaMemcpyHostToDevice,
                                 ws.copy),
                 "reference upload");
        IBS_CUDA(cudaEventRecord(ws.stageFree[slot], ws.copy), "staging event");
        slot ^= 1;
    }
    return IBS_OK;
}
} // namespace

extern "C" ibs_status ibs_scan_packed(ibs_table *t, const uint64_t *seq2bit,
                                      const uint64_t *nmask, const uint64_t *lens, uint32_t n,
                                      uint32_t W, ibs_window *rows, uint64_t cap)
{
    clear_error();
    if (!t || (n && (!lens || !seq2bit || !nmask))) {
        set_error("ibs_scan_packed: bad argument");
        return IBS_ERR_ARG;
    }
    const ibs_status lenStatus = check_contig_lengths(lens, n, "ibs_scan_packed");
    if (lenStatus != IBS_OK)
        return lenStatus;
    const uint32_t k = t->geom.k;
    if (W <= k) {
        set_error("window size " + std::to_string(W) + " must be larger than k (" +
                  std::to_string(k) + ")");
        return IBS_ERR_ARG;
    }
    const uint64_t nWin = ibs_window_count(lens, n, W, k);
    if (nWin > cap || (nWin && !rows)) {
        set_error("ibs_scan_packed: row capacity too small");
        return IBS_ERR_ARG;
    }
    if (t->device < 0 || t->device >= 16) {
        set_error("ibs_scan_packed: device ordinal beyond 15");
        return IBS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_wsMu);
    Workspace &ws = g_ws[t->device];
    DeviceGuard guard(t->device);
    if (ws.device < 0) {
        IBS_CUDA(cudaStreamCreateWithFlags(&ws.copy, cudaStreamNonBlocking), "stream create");
        IBS_CUDA(cudaStreamCreateWithFlags(&ws.comp, cudaStreamNonBlocking), "stream create");
        ws.stageBytes = 32ull << 20;
        for (int i = 0; i < 2; ++i) {
            IBS_CUDA(cudaMallocHost(&ws.stage[i], ws.stageBytes), "pinned staging");
            IBS_CUDA(cudaEventCreateWithFlags(&ws.stageFree[i], cudaEventDisableTiming),
                     "event create");
        }
        ws.device = t->device;
    }
    // the workspace's device arrays are rewritten below: wait for any work a
    // previous call left queued on its streams (a call that failed after
    // enqueueing returns without waiting)
    IBS_CUDA(cudaStreamSynchronize(ws.comp), "scan workspace");
    IBS_CUDA(cudaStreamSynchronize(ws.copy), "scan workspace");
    std::vector<uint64_t> off;
    uint64_t seqWords, maskWords;
    packed_offsets(lens, n, off, seqWords, maskWords);
    std::vector<uint64_t> lv(lens, lens + n);
    ScanPlan &p = ws.plan;
    plan_windows(p, lv, off, W, k, tuning().span_len);
    if (p.nSpans > ws.spansCap || !p.dSpans) {
        cudaFree(p.dSpans);
        p.dSpans = nullptr;
        ws.spansCap = 0;
        IBS_CUDA(cudaMalloc(&p.dSpans, std::max<uint64_t>(p.nSpans, 1) * sizeof(SegStats)),
                 "span scratch alloc");
        ws.spansCap = std::max<uint64_t>(p.nSpans, 1);
    }
    if (p.nWin + 1 > ws.winCap || !p.dWin) { // kept across calls (both streams are idle here)
        cudaFree(p.dWin);
        cudaFree(p.dSpan0);
        p.dWin = nullptr;
        p.dSpan0 = nullptr;
        ws.winCap = 0;
        IBS_CUDA(cudaMalloc(&p.dWin, (p.nWin + 1) * sizeof(WinDesc)), "plan alloc");
        IBS_CUDA(cudaMalloc(&p.dSpan0, (p.nWin + 1) * sizeof(uint32_t)), "plan alloc");
        ws.winCap = p.nWin + 1;
    }
    ibs_status s = grow(ws.dSeq, ws.seqCap, seqWords, "reference alloc");
    if (s != IBS_OK)
        return s;
    s = grow(ws.dMask, ws.maskCap, maskWords, "reference alloc");
    if (s != IBS_OK)
        return s;
    if (ws.rowsCap < nWin) {
        cudaFree(ws.dRows);
        ws.dRows = nullptr;
        ws.rowsCap = 0;
        IBS_CUDA(cudaMalloc(&ws.dRows, std::max<uint64_t>(nWin, 1) * sizeof(ibs_window)),
                 "row buffer alloc");
        ws.rowsCap = nWin;
    }
    const bool pinnedIn = is_pinned(seq2bit) && is_pinned(nmask);
    // window groups: the first 1/128 of the reference (at least 4 Mbase), so
    // that the scan starts after a short copy, then each group 1.3x the one
    // before (a copy of the next group takes no longer than the scan of the
    // current one: host-to-device bandwidth carries about 1.35x the scan's
    // bases per second) up to 1/8 of the reference
    const uint64_t totalBases = (seqWords - 1) * 32;
    const uint64_t maxGroup = std::max<uint64_t>(totalBases / 8 + 1, 16ull << 20);
    std::vector<uint64_t> gWin; // first window of each group
    {
        uint64_t lastBase = 0, size = std::max<uint64_t>(totalBases / 128 + 1, 4ull << 20);
        for (uint64_t w = 0; w < p.nWin; ++w)
            if (gWin.empty() || p.win[w].base >= lastBase + size) {
                if (!gWin.empty())
                    size = std::min<uint64_t>(maxGroup, size + size * 3 / 10);
                gWin.push_back(w);
                lastBase = p.win[w].base;
            }
        gWin.push_back(p.nWin);
    }
    const size_t G = gWin.size() - 1;
    while (ws.ev.size() < G + 1) {
        cudaEvent_t e;
        IBS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event create");
        ws.ev.push_back(e);
    }
    // the plan arrays go first, on the copy stream
    s = copy_h2d(ws, p.dWin, p.win.data(), p.nWin * sizeof(WinDesc), false);
    if (s != IBS_OK)
        return s;
    s = copy_h2d(ws, p.dSpan0, p.span0.data(), (p.nWin + 1) * sizeof(uint32_t), false);
    if (s != IBS_OK)
        return s;
    // group g copies seq words [cs_g, cs_{g+1}) and mask words [cm_g, cm_{g+1})
    std::vector<uint64_t> cs(G + 1), cm(G + 1);
    for (size_t g = 0; g < G; ++g) {
        cs[g] = g == 0 ? 0 : p.win[gWin[g]].base / 32;
        cm[g] = g == 0 ? 0 : p.win[gWin[g]].base / 64;
    }
    cs[G] = seqWords;
    cm[G] = maskWords;
    for (size_t g = 0; g < G; ++g) {
        s = copy_h2d(ws, ws.dSeq + cs[g], seq2bit + cs[g], (cs[g + 1] - cs[g]) * 8, pinnedIn);
        if (s != IBS_OK)
            return s;
        s = copy_h2d(ws, ws.dMask + cm[g], nmask + cm[g], (cm[g + 1] - cm[g]) * 8, pinnedIn);
        if (s != IBS_OK)
            return s;
        IBS_CUDA(cudaEventRecord(ws.ev[g], ws.copy), "event record");
    }
    if (G == 0)
        IBS_CUDA(cudaEventRecord(ws.ev[0], ws.copy), "event record");
    // group g's kernel waits for the copy group holding its last word
    for (size_t g = 0; g < G; ++g) {
        const WinDesc &lw = p.win[gWin[g + 1] - 1];
        const uint64_t lastBase = lw.base + (uint64_t)(lw.end - lw.start);
        const uint64_t lastWord = lastBase / 32 + 1, lastMaskWord = lastBase / 64 + 1;
        size_t need = g;
        while (need + 1 < G && (cs[need + 1] <= lastWord || cm[need + 1] <= lastMaskWord))
            ++need;
        IBS_CUDA(cudaStreamWaitEvent(ws.comp, ws.ev[need], 0), "stream wait");
        s = launch_spans(t, ws.dSeq, ws.dMask, p, p.span0[gWin[g]], p.span0[gWin[g + 1]],
                         p.dSpans, ws.comp);
        if (s != IBS_OK)
            return s;
    }
    IBS_CUDA(cudaStreamWaitEvent(ws.comp, ws.ev[G ? G - 1 : 0], 0), "stream wait");
    s = launch_finalize(p, k, ws.dRows, ws.comp);
    if (s != IBS_OK)
        return s;
    if (nWin)
        IBS_CUDA(cudaMemcpyAsync(rows, ws.dRows, nWin * sizeof(ibs_window), cudaMemcpyDeviceToHost,
                                 ws.comp),
                 "row download");
    IBS_CUDA(cudaStreamSynchronize(ws.comp), "scan");
    IBS_CUDA(cudaStreamSynchronize(ws.copy), "scan");
    return IBS_OK;
}

extern "C" ibs_status ibs_set_tuning(const ibs_tuning *t)
{
    clear_error();
    if (!t) {
        set_error("ibs_set_tuning: null");
        return IBS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_tuneMu);
    ibs_tuning n = g_tune;
    if (t->span_len) {
        if (t->span_len % 128 || t->span_len > (1u << 24)) {
            set_error("ibs_set_tuning: span_len must be a multiple of 128");
            return IBS_ERR_ARG;
        }
        n.span_len = t->span_len;
    }
    if (t->blocks_in_flight) {
        if (t->blocks_in_flight != 1 && t->blocks_in_flight != 2 && t->blocks_in_flight != 4 &&
            t->blocks_in_flight != 8) {
            set_error("ibs_set_tuning: blocks_in_flight must be 1, 2, 4 or 8");
            return IBS_ERR_ARG;
        }
        n.blocks_in_flight = t->blocks_in_flight;
    }
    if (t->block_threads) {
        if (t->block_threads != 128 && t->block_threads != 256 && t->block_threads != 512) {
            set_error("ibs_set_tuning: block_threads must be 128, 256 or 512");
            return IBS_ERR_ARG;
        }
        n.block_threads = t->block_threads;
    }
    if (t->ctas_per_sm)
        n.ctas_per_sm = std::min<uint32_t>(t->ctas_per_sm, 64);
    if (t->keys_per_bucket > 0)
        n.keys_per_bucket = t->keys_per_bucket;
    if (t->table_format)
        n.table_format = t->table_format == 0xffffffffu ? 0 : t->table_format;
    if (t->panel_pass_mb)
        n.panel_pass_mb = t->panel_pass_mb == 0xffffffffu ? 0 : t->panel_pass_mb;
    if (t->panel_span_len) {
        if (t->panel_span_len % 128 || t->panel_span_len > (1u << 24)) {
            set_error("ibs_set_tuning: panel_span_len must be a multiple of 128");
            return IBS_ERR_ARG;
        }
        n.panel_span_len = t->panel_span_len;
    }
    if (t->panel_ctas_per_sm)
        n.panel_ctas_per_sm = std::min<uint32_t>(t->panel_ctas_per_sm, 8);
    if (t->panel_keys_per_bucket > 0) {
        if (t->panel_keys_per_bucket > 5.0) {
            set_error("ibs_set_tuning: panel_keys_per_bucket must be at most 5 (slots per bucket)");
            return IBS_ERR_ARG;
        }
        n.panel_keys_per_bucket = t->panel_keys_per_bucket;
    }
    if (t->panel_blocks_in_flight) {
        if (t->panel_blocks_in_flight != 2 && t->panel_blocks_in_flight != 4) {
            set_error("ibs_set_tuning: panel_blocks_in_flight must be 2 or 4");
            return IBS_ERR_ARG;
        }
        n.panel_blocks_in_flight = t->panel_blocks_in_flight;
    }
    g_tune = n;
    return IBS_OK;
}

extern "C" void ibs_get_tuning(ibs_tuning *t)
{
    if (t) {
        std::lock_guard<std::mutex> lock(g_tuneMu);
        *t = g_tune;
    }
}
