// The reference mapper (fastibsmapper): for every base of every contig, how
// many k-mers of the sample cover it -- the number of k-mer starts s in
// [i - k + 1, i] whose canonical k-mer is in the table (KmerDatabase::
// getMappingFromSequence and its GPU consumer, src/KmerDatabase.hpp:774-801,
// :1544-1581). The reference accumulates +1/-1 into a per-contig difference
// array and prefix-sums it; here a warp probes 32 starts per step and each
// lane counts the hits among the k starts that cover its base straight from
// the current and previous hit ballots (k <= 32; three ballots for the
// wide-key tables of 33 <= k <= 64). The output text (per
// contig: the id, a newline, the coverage values joined by commas, a
// newline; src/KmerDatabase.hpp:754-772, :1195-1203) is also written on the
// device: each 8192-value tile is sized, the tile offsets are summed on the
// host, and a second pass ranks each thread's characters with a block scan.
#include "ibs_internal.cuh"
#include "scan_device.cuh"

#include <cub/block/block_scan.cuh>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace ibs {
namespace map {

constexpr uint32_t kSpan = 4096;       // bases per warp task
constexpr uint32_t kThreads = 256;
constexpr uint32_t kPerThread = 32;
constexpr uint32_t kTile = kThreads * kPerThread; // coverage values per text tile

struct Span {
    uint64_t base;   // packed base offset of the contig's first base
    uint64_t out;    // coverage index of the contig's first base
    uint32_t a, b;   // bases [a, b) of the contig
    uint32_t nPos;   // k-mer starts of the contig
    uint32_t pad;
};

template <uint32_t FMT>
__device__ __forceinline__ bool hit_at(const TableView &t, const uint64_t *__restrict__ seq,
                                       const uint64_t *__restrict__ mask, const Span &sp, uint32_t s,
                                       uint32_t k, uint64_t kmask, uint64_t kbits)
{
    if (s >= sp.nPos)
        return false;
    bool acgt;
    const uint64_t code = dev::canonical_at(seq, mask, sp.base + s, k, kmask, kbits, acgt);
    return acgt && table_lookup<FMT>(t, code);
}

template <uint32_t FMT>
__global__ void __launch_bounds__(256) k_map_spans(TableView t, const uint64_t *__restrict__ seq,
                                                   const uint64_t *__restrict__ mask,
                                                   const Span *__restrict__ spans, uint64_t nSpans,
                                                   uint8_t *__restrict__ cov)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = t.g.k;
    const uint64_t kmask = key_mask(2 * k);
    const uint64_t kbits = key_mask(k);
    for (uint64_t i = warp; i < nSpans; i += nWarps) {
        const Span sp = spans[i];
        // hits of the 32 starts before the span (the k-1 that cover its first bases)
        uint32_t prev = 0;
        if (sp.a >= 32)
            prev = __ballot_sync(dev::FULL_MASK, hit_at<FMT>(t, seq, mask, sp, sp.a - 32 + lane, k, kmask, kbits));
        for (uint32_t p = sp.a; p < sp.b; p += 32) {
            const uint32_t H =
                __ballot_sync(dev::FULL_MASK, hit_at<FMT>(t, seq, mask, sp, p + lane, k, kmask, kbits));
            // bit j of M: start p - 32 + j; base p + lane is covered by the
            // starts p + lane - k + 1 .. p + lane, bits 33 + lane - k .. 32 + lane
            const uint64_t M = ((uint64_t)H << 32) | prev;
            if (p + lane < sp.b)
                cov[sp.out + p + lane] = (uint8_t)__popcll((M >> (33 + lane - k)) & kbits);
            prev = H;
        }
    }
}

// The same for a wide-key table (33 <= k <= 64): a base is covered by up to
// 64 starts, so each lane counts from the current ballot and the two before
// it (starts p - 64 .. p + 31). The reference's string-path mapper
// (getMappingFromSequenceLegacy, src/KmerDatabase.hpp:803-848) adds 1 to the
// k bases of every start whose canonical k-mer string the database holds.
// Every lane of the warp calls it (the lookup is warp-cooperative).
__device__ __forceinline__ bool hit_at_wide(const wide::View &t, const uint64_t *__restrict__ seq,
                                            const uint64_t *__restrict__ mask, const Span &sp, uint32_t s, uint32_t k,
                                            uint32_t lane)
{
    bool acgt = false;
    uint64_t lo = 0, hi = 0;
    if (s < sp.nPos)
        wide::canonical_at(seq, mask, sp.base + s, k, acgt, lo, hi);
    return wide::lookup_warp(t, lo, hi, s < sp.nPos && acgt, lane);
}

__global__ void __launch_bounds__(256) k_map_spans_wide(wide::View t, const uint64_t *__restrict__ seq,
                                                        const uint64_t *__restrict__ mask,
                                                        const Span *__restrict__ spans, uint64_t nSpans,
                                                        uint8_t *__restrict__ cov)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t k = t.k;
    const uint64_t kbits = key_mask(k);
    for (uint64_t i = warp; i < nSpans; i += nWarps) {
        const Span sp = spans[i];
        // hits of the 64 starts before the span (spans start at 0 or at a
        // multiple of kSpan >= 64)
        uint32_t prev1 = 0, prev2 = 0; // starts p - 32 .. p - 1 and p - 64 .. p - 33
        if (sp.a >= 64) {
            prev2 = __ballot_sync(dev::FULL_MASK, hit_at_wide(t, seq, mask, sp, sp.a - 64 + lane, k, lane));
            prev1 = __ballot_sync(dev::FULL_MASK, hit_at_wide(t, seq, mask, sp, sp.a - 32 + lane, k, lane));
        }
        for (uint32_t p = sp.a; p < sp.b; p += 32) {
            const uint32_t H = __ballot_sync(dev::FULL_MASK, hit_at_wide(t, seq, mask, sp, p + lane, k, lane));
            // bit j of (H : prev1 : prev2) is start p - 64 + j; base p + lane
            // is covered by bits 65 + lane - k .. 64 + lane (1 <= low <= 96)
            const uint64_t lowWord = ((uint64_t)prev1 << 32) | prev2;
            const uint32_t low = 65 + lane - k;
            const uint64_t x = low >= 64 ? ((uint64_t)H >> (low - 64))
                                         : ((lowWord >> low) | ((uint64_t)H << (64 - low)));
            if (p + lane < sp.b)
                cov[sp.out + p + lane] = (uint8_t)__popcll(x & kbits);
            prev2 = prev1;
            prev1 = H;
        }
    }
}

struct Tile {
    uint64_t first;  // coverage index of the tile's first value
    uint32_t n;      // values (<= kTile)
    uint32_t last;   // 1 when the tile ends its contig (its last value ends the line)
};

__device__ __forceinline__ uint32_t chars_of(uint8_t v) { return v >= 10 ? 3u : 2u; } // digits + separator

__global__ void k_text_sizes(const uint8_t *__restrict__ cov, const Tile *__restrict__ tiles, uint64_t nTiles,
                             uint64_t *__restrict__ sizes)
{
    __shared__ uint32_t warpSum[kThreads / 32];
    for (uint64_t t = blockIdx.x; t < nTiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        uint32_t c = 0;
        for (uint32_t i = threadIdx.x; i < tl.n; i += kThreads)
            c += chars_of(cov[tl.first + i]);
        for (int o = 16; o; o >>= 1)
            c += __shfl_xor_sync(0xffffffffu, c, o);
        if ((threadIdx.x & 31) == 0)
            warpSum[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t s = 0;
            for (uint32_t w = 0; w < kThreads / 32; ++w)
                s += warpSum[w];
            sizes[t] = s;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads) k_text_write(const uint8_t *__restrict__ cov,
                                                         const Tile *__restrict__ tiles, uint64_t nTiles,
                                                         const uint64_t *__restrict__ offsets,
                                                         char *__restrict__ text)
{
    using Scan = cub::BlockScan<uint32_t, kThreads>;
    __shared__ typename Scan::TempStorage tmp;
    for (uint64_t t = blockIdx.x; t < nTiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        const uint32_t i0 = threadIdx.x * kPerThread;
        const uint32_t i1 = min(i0 + kPerThread, tl.n);
        uint32_t mine = 0;
        for (uint32_t i = i0; i < i1; ++i)
            mine += chars_of(cov[tl.first + i]);
        uint32_t before = 0;
        Scan(tmp).ExclusiveSum(mine, before);
        char *o = text + offsets[t] + before;
        for (uint32_t i = i0; i < i1; ++i) {
            const uint8_t v = cov[tl.first + i];
            if (v >= 10)
                *o++ = (char)('0' + v / 10);
            *o++ = (char)('0' + v % 10);
            *o++ = (tl.last && i + 1 == tl.n) ? '\n' : ',';
        }
        __syncthreads(); // tmp is reused by the next tile
    }
}

int grid_for(uint64_t n, uint64_t perBlock)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + perBlock - 1) / perBlock, (uint64_t)sms * 8));
}

// Per-base coverage of every contig into dCov (sum of the lengths).
ibs_status coverage_device(ibs_table *t, const ibs_reference *ref, uint8_t *dCov)
{
    const uint32_t k = t->geom.k;
    std::vector<Span> spans;
    uint64_t out = 0;
    for (size_t c = 0; c < ref->lens.size(); ++c) {
        const uint64_t len = ref->lens[c];
        if (len >= (1ull << 32)) {
            set_error("mapper: contigs of 2^32 bases or more are not supported");
            return IBS_ERR_CAPACITY;
        }
        const uint32_t nPos = len >= k ? (uint32_t)(len - k + 1) : 0;
        for (uint64_t a = 0; a < len; a += kSpan)
            spans.push_back(Span{ref->baseOff[c], out, (uint32_t)a, (uint32_t)std::min<uint64_t>(a + kSpan, len),
                                 nPos, 0});
        out += len;
    }
    if (spans.empty())
        return IBS_OK;
    Span *dSpans = nullptr;
    IBS_CUDA(cudaMalloc(&dSpans, spans.size() * sizeof(Span)), "mapper span alloc");
    std::unique_ptr<Span, cudaError_t (*)(void *)> g(dSpans, cudaFree);
    IBS_CUDA(cudaMemcpy(dSpans, spans.data(), spans.size() * sizeof(Span), cudaMemcpyHostToDevice),
             "mapper span upload");
    const int grid = grid_for(spans.size(), 8); // 8 warps per block
    const TableView v = t->view();
    if (t->geom.format == FMT_WIDE)
        k_map_spans_wide<<<grid, 256>>>(t->wide, ref->dSeq, ref->dMask, dSpans, spans.size(), dCov);
    else if (t->geom.format == FMT_B8X32)
        k_map_spans<FMT_B8X32><<<grid, 256>>>(v, ref->dSeq, ref->dMask, dSpans, spans.size(), dCov);
    else if (t->geom.format == FMT_MZ8)
        k_map_spans<FMT_MZ8><<<grid, 256>>>(v, ref->dSeq, ref->dMask, dSpans, spans.size(), dCov);
    else if (t->geom.format == FMT_MZ6)
        k_map_spans<FMT_MZ6><<<grid, 256>>>(v, ref->dSeq, ref->dMask, dSpans, spans.size(), dCov);
    else
        k_map_spans<FMT_B6X40><<<grid, 256>>>(v, ref->dSeq, ref->dMask, dSpans, spans.size(), dCov);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "mapper launch");
    IBS_CUDA(cudaDeviceSynchronize(), "mapper");
    return IBS_OK;
}

ibs_status check_args(ibs_table *t, const ibs_reference *ref, const char *what)
{
    if (!t || !ref) {
        set_error(std::string(what) + ": bad argument");
        return IBS_ERR_ARG;
    }
    if (t->device != ref->device) {
        set_error(std::string(what) + ": the table and the reference are on different devices");
        return IBS_ERR_ARG;
    }
    return IBS_OK;
}

} // namespace map
} // namespace ibs

using namespace ibs;
using namespace ibs::map;

extern "C" ibs_status ibs_map_coverage(ibs_table *t, ibs_reference *ref, uint8_t *coverage, uint64_t cap)
{
    clear_error();
    ibs_status s = check_args(t, ref, "ibs_map_coverage");
    if (s != IBS_OK)
        return s;
    uint64_t total = 0;
    for (uint64_t l : ref->lens)
        total += l;
    if (total > cap || (total && !coverage)) {
        set_error("ibs_map_coverage: capacity below the reference's length");
        return IBS_ERR_ARG;
    }
    if (!total)
        return IBS_OK;
    DeviceGuard guard(t->device);
    uint8_t *dCov = nullptr;
    IBS_CUDA(cudaMalloc(&dCov, total), "coverage alloc");
    std::unique_ptr<uint8_t, cudaError_t (*)(void *)> g(dCov, cudaFree);
    s = coverage_device(t, ref, dCov);
    if (s != IBS_OK)
        return s;
    IBS_CUDA(cudaMemcpy(coverage, dCov, total, cudaMemcpyDeviceToHost), "coverage download");
    return IBS_OK;
}

extern "C" ibs_status ibs_map_text(ibs_table *t, ibs_reference *ref, const char *const *ids, char **text,
                                   uint64_t *n_bytes)
{
    clear_error();
    ibs_status s = check_args(t, ref, "ibs_map_text");
    if (s != IBS_OK)
        return s;
    if (!text || !n_bytes) {
        set_error("ibs_map_text: bad argument");
        return IBS_ERR_ARG;
    }
    *text = nullptr;
    *n_bytes = 0;
    const size_t nc = ref->lens.size();
    std::vector<std::string> names(nc);
    for (size_t c = 0; c < nc; ++c)
        names[c] = ids ? std::string(ids[c] ? ids[c] : "") : (c < ref->ids.size() ? ref->ids[c] : "");
    uint64_t total = 0;
    for (uint64_t l : ref->lens)
        total += l;
    // tiles of each contig's values; the last one of a contig ends its line
    std::vector<Tile> tiles;
    std::vector<size_t> firstTile(nc + 1);
    uint64_t first = 0;
    for (size_t c = 0; c < nc; ++c) {
        firstTile[c] = tiles.size();
        const uint64_t len = ref->lens[c];
        for (uint64_t a = 0; a < len; a += kTile)
            tiles.push_back(Tile{first + a, (uint32_t)std::min<uint64_t>(kTile, len - a),
                                 a + kTile >= len ? 1u : 0u});
        first += len;
    }
    firstTile[nc] = tiles.size();
    const uint64_t nTiles = tiles.size();
    DeviceGuard guard(t->device);
    uint8_t *dCov = nullptr;
    Tile *dTiles = nullptr;
    uint64_t *dSizes = nullptr;
    char *dText = nullptr;
    auto freeAll = [&]() {
        cudaFree(dCov);
        cudaFree(dTiles);
        cudaFree(dSizes);
        cudaFree(dText);
    };
    struct Guard {
        decltype(freeAll) &f;
        ~Guard() { f(); }
    } g{freeAll};
    IBS_CUDA(cudaMalloc(&dCov, std::max<uint64_t>(total, 1)), "coverage alloc");
    s = coverage_device(t, ref, dCov);
    if (s != IBS_OK)
        return s;
    std::vector<uint64_t> sizes(nTiles);
    if (nTiles) {
        IBS_CUDA(cudaMalloc(&dTiles, nTiles * sizeof(Tile)), "text tiles alloc");
        IBS_CUDA(cudaMalloc(&dSizes, nTiles * 8), "text tiles alloc");
        IBS_CUDA(cudaMemcpy(dTiles, tiles.data(), nTiles * sizeof(Tile), cudaMemcpyHostToDevice), "text tiles");
        k_text_sizes<<<grid_for(nTiles, 1), kThreads>>>(dCov, dTiles, nTiles, dSizes);
        IBS_LAUNCHED();
        IBS_CUDA(cudaGetLastError(), "text size launch");
        IBS_CUDA(cudaMemcpy(sizes.data(), dSizes, nTiles * 8, cudaMemcpyDeviceToHost), "text sizes");
    }
    // layout: per contig "<id>\n" then its values; a contig without bases
    // still ends its (empty) value line
    std::vector<uint64_t> headerAt(nc), offsets(nTiles);
    uint64_t pos = 0;
    for (size_t c = 0; c < nc; ++c) {
        headerAt[c] = pos;
        pos += names[c].size() + 1;
        if (firstTile[c] == firstTile[c + 1])
            pos += 1;
        for (size_t i = firstTile[c]; i < firstTile[c + 1]; ++i) {
            offsets[i] = pos;
            pos += sizes[i];
        }
    }
    const uint64_t n = pos;
    char *host = nullptr;
    IBS_CUDA(cudaMallocHost(&host, std::max<uint64_t>(n, 1)), "text pinned alloc");
    if (nTiles) {
        cudaError_t e = cudaMalloc(&dText, n);
        uint64_t *dOff = dSizes; // reuse: the sizes are on the host now
        if (e == cudaSuccess)
            e = cudaMemcpy(dOff, offsets.data(), nTiles * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) {
            k_text_write<<<grid_for(nTiles, 1), kThreads>>>(dCov, dTiles, nTiles, dOff, dText);
            IBS_LAUNCHED();
            e = cudaGetLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpy(host, dText, n, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            cudaFreeHost(host);
            return cuda_fail(e, "text write");
        }
    }
    for (size_t c = 0; c < nc; ++c) {
        memcpy(host + headerAt[c], names[c].data(), names[c].size());
        host[headerAt[c] + names[c].size()] = '\n';
        if (firstTile[c] == firstTile[c + 1])
            host[headerAt[c] + names[c].size() + 1] = '\n';
    }
    *text = host;
    *n_bytes = n;
    return IBS_OK;
}

extern "C" void ibs_map_text_free(char *text)
{
    if (text)
        cudaFreeHost(text);
}
