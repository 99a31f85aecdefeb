// ibs_scan_noalloc: the window scan with no memory allocation.
//
// Some callers cannot allocate device memory when they scan: a serving
// process that has handed all of the GPU's free memory to its own pool, a
// host that must keep its device allocations fixed after start-up, or a
// latency-bound loop for which cudaMalloc (which may synchronize the device)
// is not acceptable. This entry point serves them: the caller passes the
// table, the packed reference and the row buffer, all already on the device,
// and the scan's scratch (a per-contig window table and one summary per
// span) lives in the fixed array g_scratch below, which every GPU that loads
// the library holds until the process exits.
//
// The kernels are the scan of ibs_scan.cu with its per-window plan replaced
// by per-contig window arithmetic, so nothing per window has to be uploaded.
#include "ibs_internal.cuh"
#include "scan_device.cuh"

#include <cub/block/block_scan.cuh>

#include <mutex>

namespace ibs {
namespace noalloc {

constexpr uint64_t kScratchBytes = IBS_NOALLOC_SCRATCH_BYTES; // per device
constexpr uint32_t kSpanLen = 4096;
constexpr int kNB = 4;
constexpr int kMaxDevices = 64;

// The scratch of every call on this device. Host code must not pass this
// name to a kernel (on the host it is only a stand-in for the symbol); it
// uses the address cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct ContigDesc {
    uint64_t base, len, win0, span0; // packed base offset, length, first window, first span
};

struct ContigWin {
    uint64_t nWin, nFull, spw; // windows; the first nFull have W bases; spans of such a window
};

// Windows of a contig of L bases: chunkSequences (src/Utils.hpp:296-327)
// cuts [j, min(j+W, L)) for j = 0, W-k, ...; window i is full-length while
// i(W-k) + W <= L, and only the last few are shorter.
IBS_HD ContigWin contig_windows(uint64_t L, uint32_t W, uint32_t k)
{
    ContigWin r;
    const uint64_t step = (uint64_t)W - k;
    r.nWin = L ? (L + step - 1) / step : 0;
    r.nFull = L >= W ? (L - W) / step + 1 : 0;
    r.spw = ((uint64_t)W - k + 1 + kSpanLen - 1) / kSpanLen;
    return r;
}

IBS_HD uint64_t window_npos(uint64_t L, uint64_t i, uint32_t W, uint32_t k)
{
    const uint64_t j = i * ((uint64_t)W - k);
    const uint64_t nb = j + W <= L ? (uint64_t)W : L - j;
    return nb >= k ? nb - k + 1 : 0;
}

IBS_HD uint64_t spans_of(uint64_t npos) { return (npos + kSpanLen - 1) / kSpanLen; }

IBS_HD uint64_t contig_spans(uint64_t L, uint32_t W, uint32_t k)
{
    const ContigWin cw = contig_windows(L, W, k);
    uint64_t s = cw.nFull * cw.spw;
    for (uint64_t i = cw.nFull; i < cw.nWin; ++i)
        s += spans_of(window_npos(L, i, W, k));
    return s;
}

// Per-contig descriptors from the contig lengths (one block; running carry
// over chunks of 1024 contigs).
__global__ void __launch_bounds__(1024) k_na_desc(const uint64_t *__restrict__ lens, uint32_t n,
                                                  uint32_t W, uint32_t k, ContigDesc *__restrict__ cd)
{
    using Scan = cub::BlockScan<uint64_t, 1024>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint64_t carry[3];
    if (threadIdx.x == 0)
        carry[0] = carry[1] = carry[2] = 0;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < n; c0 += 1024) {
        const uint32_t c = c0 + threadIdx.x;
        const uint64_t L = c < n ? lens[c] : 0;
        const uint64_t a = c < n ? round_up64(L) : 0;
        const uint64_t b = c < n ? contig_windows(L, W, k).nWin : 0;
        const uint64_t s = c < n ? contig_spans(L, W, k) : 0;
        uint64_t ea, eb, es, ta, tb, ts;
        Scan(tmp).ExclusiveSum(a, ea, ta);
        __syncthreads();
        Scan(tmp).ExclusiveSum(b, eb, tb);
        __syncthreads();
        Scan(tmp).ExclusiveSum(s, es, ts);
        if (c < n) {
            ContigDesc d;
            d.base = carry[0] + ea;
            d.len = L;
            d.win0 = carry[1] + eb;
            d.span0 = carry[2] + es;
            cd[c] = d;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry[0] += ta;
            carry[1] += tb;
            carry[2] += ts;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ uint32_t last_le(const ContigDesc *cd, uint32_t n, uint64_t v, bool bySpan)
{
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        const uint64_t x = bySpan ? cd[mid].span0 : cd[mid].win0;
        if (x <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

template <uint32_t FMT, int NB>
__global__ void __launch_bounds__(256) k_na_spans(TableView t, const uint64_t *__restrict__ seq,
                                                  const uint64_t *__restrict__ mask,
                                                  const ContigDesc *__restrict__ cd, uint32_t n,
                                                  uint32_t W, uint64_t nSpans,
                                                  SegStats *__restrict__ out)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = t.g.k;
    const uint64_t kmask = key_mask(2 * k);
    const uint64_t kbits = (1ull << k) - 1;
    for (uint64_t s = warp; s < nSpans; s += nWarps) {
        const uint32_t c = last_le(cd, n, s, true);
        const uint64_t L = cd[c].len;
        const ContigWin cw = contig_windows(L, W, k);
        uint64_t sc = s - cd[c].span0, i, nPos;
        if (sc < cw.nFull * cw.spw) {
            i = sc / cw.spw;
            sc -= i * cw.spw;
            nPos = (uint64_t)W - k + 1;
        } else {
            sc -= cw.nFull * cw.spw;
            i = cw.nFull;
            for (;;) {
                nPos = window_npos(L, i, W, k);
                const uint64_t sp = spans_of(nPos);
                if (sc < sp)
                    break;
                sc -= sp;
                ++i;
            }
        }
        const uint64_t base = cd[c].base + i * ((uint64_t)W - k);
        const uint32_t p0 = (uint32_t)sc * kSpanLen;
        const uint32_t p1 = (uint32_t)(p0 + kSpanLen < nPos ? p0 + kSpanLen : nPos);
        dev::LaneFold fold;
        for (uint32_t p = p0; p < p1; p += 32 * NB) {
            uint4 v0[NB], v1[NB];
            uint64_t code[NB], fp[NB];
            bool valid[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const uint32_t q = p + 32 * b + lane;
                const bool inSpan = q < p1;
                const uint64_t G = base + (inSpan ? q : p0);
                bool acgt;
                code[b] = dev::canonical_at(seq, mask, G, k, kmask, kbits, acgt);
                valid[b] = inSpan && acgt;
                const uint64_t h = perm_hash(code[b], t.g.bits);
                const uint64_t r = bucket_of(h, t.g);
                fp[b] = fp_of(h, t.g);
                if (valid[b] && !is_mz(FMT)) {
                    v0[b] = __ldg(t.buckets + 2 * r);
                    v1[b] = __ldg(t.buckets + 2 * r + 1);
                } else {
                    v0[b] = make_uint4(0, 0, 0, 0);
                    v1[b] = make_uint4(0, 0, 0, 0);
                }
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                bool hit = false;
                if (valid[b]) {
                    if constexpr (FMT == FMT_MZ8 || FMT == FMT_MZ6) {
                        // minimizer table: each lane finds its k-mer's minimizer on its own
                        hit = table_lookup<FMT>(t, code[b]);
                    } else {
                        const uint32_t m = bucket_match<FMT>(v0[b], v1[b], fp[b]);
                        hit = m == 1u || (m == 2u && stash_lookup(t, code[b]));
                    }
                }
                const uint32_t V = __ballot_sync(dev::FULL_MASK, valid[b]);
                const uint32_t H = __ballot_sync(dev::FULL_MASK, hit);
                fold.push(V, H, lane, (int)k);
            }
        }
        const SegStats acc = fold.finish((int)k);
        if (lane == 0)
            out[s] = acc;
    }
}

__global__ void k_na_finalize(const ContigDesc *__restrict__ cd, uint32_t n, uint32_t W, uint32_t k,
                              uint64_t nWin, const SegStats *__restrict__ spans,
                              ibs_window *__restrict__ rows)
{
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < nWin;
         w += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = last_le(cd, n, w, false);
        const uint64_t L = cd[c].len;
        const ContigWin cw = contig_windows(L, W, k);
        const uint64_t i = w - cd[c].win0;
        uint64_t first, cnt;
        if (i < cw.nFull) {
            first = cd[c].span0 + i * cw.spw;
            cnt = cw.spw;
        } else {
            first = cd[c].span0 + cw.nFull * cw.spw;
            for (uint64_t j = cw.nFull; j < i; ++j)
                first += spans_of(window_npos(L, j, W, k));
            cnt = spans_of(window_npos(L, i, W, k));
        }
        SegStats acc = seg_empty();
        for (uint64_t s = first; s < first + cnt; ++s)
            acc = seg_combine(acc, spans[s], (int)k);
        const uint64_t j0 = i * ((uint64_t)W - k);
        WindowRow row;
        row.start = (int32_t)j0;
        row.end = (int32_t)(j0 + W <= L ? j0 + W : L);
        seg_finish(acc, (int)k, row);
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

// One-time set-up per device: the device address of g_scratch, looked up
// with that device current.
std::mutex g_mu;
void *g_ptr[kMaxDevices] = {};

ibs_status scratch_address(int device, unsigned char **out)
{
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess)
            return cuda_fail(e, "ibs_scan_noalloc scratch address");
        g_ptr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_ptr[device]);
    return IBS_OK;
}

uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

} // namespace noalloc
} // namespace ibs

using namespace ibs;
using namespace ibs::noalloc;

extern "C" ibs_status ibs_scan_noalloc(ibs_table *t, const uint64_t *seq2bit_dev,
                                       const uint64_t *nmask_dev, const uint64_t *lens,
                                       uint32_t n_contigs, uint32_t W, ibs_window *rows_dev,
                                       uint64_t cap, void *stream)
{
    clear_error();
    if (!t || (n_contigs && (!lens || !seq2bit_dev || !nmask_dev))) {
        set_error("ibs_scan_noalloc: bad argument");
        return IBS_ERR_ARG;
    }
    if (t->geom.format != FMT_B8X32 && t->geom.format != FMT_B6X40 && !is_mz(t->geom.format)) {
        set_error(t->geom.format == FMT_WIDE ? "ibs_scan_noalloc: wide-key tables (k > 32) take ibs_scan"
                                             : "ibs_scan_noalloc: unknown table format");
        return IBS_ERR_UNSUPPORTED;
    }
    const uint32_t k = t->geom.k;
    if (W <= k) {
        set_error("window size " + std::to_string(W) + " must be larger than k (" +
                  std::to_string(k) + ")");
        return IBS_ERR_ARG;
    }
    if (t->device < 0 || t->device >= kMaxDevices) {
        set_error("ibs_scan_noalloc: device ordinal out of range");
        return IBS_ERR_ARG;
    }
    ibs_status cs = check_contig_lengths(lens, n_contigs, "ibs_scan_noalloc");
    if (cs != IBS_OK)
        return cs;
    uint64_t nWin = 0, nSpans = 0;
    for (uint32_t c = 0; c < n_contigs; ++c) {
        nWin += contig_windows(lens[c], W, k).nWin;
        nSpans += contig_spans(lens[c], W, k);
    }
    // the scratch limit first: a scan beyond it is refused whatever the
    // caller's buffers hold
    const uint64_t offDesc = align256((uint64_t)n_contigs * 8);
    const uint64_t offSpans = offDesc + align256((uint64_t)n_contigs * sizeof(ContigDesc));
    const uint64_t need = offSpans + nSpans * sizeof(SegStats);
    if (need > kScratchBytes) {
        set_error("ibs_scan_noalloc: this scan needs " + std::to_string(need) +
                  " bytes of scratch; the fixed maximum is " + std::to_string(kScratchBytes) +
                  " bytes (about " + std::to_string((kScratchBytes / sizeof(SegStats)) * kSpanLen / 1000000) +
                  " Mbp of reference in windows of " + std::to_string(W) +
                  "); use ibs_scan_async for larger references");
        return IBS_ERR_CAPACITY;
    }
    if (nWin > cap || (nWin && !rows_dev)) {
        set_error("ibs_scan_noalloc: row capacity " + std::to_string(cap) + " < " +
                  std::to_string(nWin) + " windows");
        return IBS_ERR_ARG;
    }
    if (nWin == 0)
        return IBS_OK;
    DeviceGuard guard(t->device);
    unsigned char *scratch = nullptr;
    ibs_status s = scratch_address(t->device, &scratch);
    if (s != IBS_OK)
        return s;
    cudaStream_t st = (cudaStream_t)stream;
    uint64_t *dLens = reinterpret_cast<uint64_t *>(scratch);
    ContigDesc *dDesc = reinterpret_cast<ContigDesc *>(scratch + offDesc);
    SegStats *dSpans = reinterpret_cast<SegStats *>(scratch + offSpans);
    IBS_CUDA(cudaMemcpyAsync(dLens, lens, (uint64_t)n_contigs * 8, cudaMemcpyHostToDevice, st),
             "ibs_scan_noalloc lengths");
    k_na_desc<<<1, 1024, 0, st>>>(dLens, n_contigs, W, k, dDesc);
    IBS_LAUNCHED();
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (nSpans) {
        const uint64_t want = (nSpans + 7) / 8;
        const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 8));
        if (t->geom.format == FMT_B8X32)
            k_na_spans<FMT_B8X32, kNB><<<grid, 256, 0, st>>>(t->view(), seq2bit_dev, nmask_dev, dDesc,
                                                             n_contigs, W, nSpans, dSpans);
        else if (t->geom.format == FMT_MZ8)
            k_na_spans<FMT_MZ8, kNB><<<grid, 256, 0, st>>>(t->view(), seq2bit_dev, nmask_dev, dDesc,
                                                           n_contigs, W, nSpans, dSpans);
        else if (t->geom.format == FMT_MZ6)
            k_na_spans<FMT_MZ6, kNB><<<grid, 256, 0, st>>>(t->view(), seq2bit_dev, nmask_dev, dDesc,
                                                           n_contigs, W, nSpans, dSpans);
        else
            k_na_spans<FMT_B6X40, kNB><<<grid, 256, 0, st>>>(t->view(), seq2bit_dev, nmask_dev, dDesc,
                                                             n_contigs, W, nSpans, dSpans);
        IBS_LAUNCHED();
    }
    const uint64_t want = (nWin + 255) / 256;
    const int grid = (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 8));
    k_na_finalize<<<grid, 256, 0, st>>>(dDesc, n_contigs, W, k, nWin, dSpans, rows_dev);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "ibs_scan_noalloc launch");
    return IBS_OK;
}
