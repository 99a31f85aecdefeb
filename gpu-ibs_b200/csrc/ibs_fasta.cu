// FASTA text to a device-resident packed reference: the reference's
// readSequenceFile for FASTA (src/Utils.hpp:170-255) and its packWindow
// (src/gpu/EncodeProbeCore.hpp:157-186) applied per contig, with the bulk of
// the work -- dropping line breaks and packing every base -- on the device.
//
// Record semantics follow the reference's reader: the text must start with
// '>'; lines split on '\n' only (a '\r' stays and packs as a non-ACGT base);
// a header is a line whose first byte is '>', its id the rest of that line;
// every other line is sequence; a record with no sequence bytes is dropped
// (so of two consecutive headers only the second names the sequence after
// them). FASTQ text is refused here (its quality lines are read on the host).
//
// The text is uploaded through the library's pinned staging slots: a few
// host threads each copy every T-th 16 MiB chunk into one of their two slots
// and issue its copy to the device on their own stream, and list the header
// starts (a '>' at a line start) of that chunk on the way. The host cuts each
// record's body into tiles. The device counts the sequence bytes
// of every tile; the host turns the counts into contig lengths and each
// tile's output base offset in the packed layout; the device then moves
// every tile through shared memory, ranks its sequence bytes with a block
// scan and ORs 2-bit codes and N-mask bits into the zeroed packed words.
#include "ibs_internal.cuh"

#include <cub/block/block_scan.cuh>

#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace ibs {
namespace fasta {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kBytesPerThread = 32;
constexpr uint32_t kTile = kThreads * kBytesPerThread; // 8192 bytes

struct Tile {
    uint64_t start;  // first byte of the tile in the text
    uint32_t len;    // bytes (<= kTile)
    uint32_t body;   // record body it belongs to
};

__global__ void k_count_tiles(const uint8_t *__restrict__ text, const Tile *__restrict__ tiles, uint64_t nTiles,
                              uint32_t *__restrict__ counts)
{
    for (uint64_t t = blockIdx.x; t < nTiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        uint32_t c = 0;
        for (uint32_t i = threadIdx.x; i < tl.len; i += blockDim.x)
            c += text[tl.start + i] != '\n' ? 1u : 0u;
        for (int o = 16; o; o >>= 1)
            c += __shfl_xor_sync(0xffffffffu, c, o);
        __shared__ uint32_t warpSum[kThreads / 32];
        if ((threadIdx.x & 31) == 0)
            warpSum[threadIdx.x >> 5] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t s = 0;
            for (uint32_t w = 0; w < kThreads / 32; ++w)
                s += warpSum[w];
            counts[t] = s;
        }
        __syncthreads();
    }
}

// 2-bit code of a base byte (A/a 0, C/c 1, G/g 2, T/t 3), 4 for anything else.
__device__ __forceinline__ uint32_t base_code(uint8_t b)
{
    switch (b | 0x20) {
    case 'a': return 0;
    case 'c': return 1;
    case 'g': return 2;
    case 't': return 3;
    default: return 4;
    }
}

__global__ void __launch_bounds__(kThreads) k_pack_tiles(const uint8_t *__restrict__ text,
                                                         const Tile *__restrict__ tiles, uint64_t nTiles,
                                                         const uint64_t *__restrict__ tileOut,
                                                         unsigned long long *__restrict__ seq,
                                                         unsigned long long *__restrict__ mask)
{
    using Scan = cub::BlockScan<uint32_t, kThreads>;
    __shared__ typename Scan::TempStorage scanTmp;
    __shared__ uint8_t buf[kTile];
    for (uint64_t t = blockIdx.x; t < nTiles; t += gridDim.x) {
        const Tile tl = tiles[t];
        for (uint32_t i = threadIdx.x; i < kTile; i += kThreads)
            buf[i] = i < tl.len ? text[tl.start + i] : (uint8_t)'\n';
        __syncthreads();
        const uint8_t *mine = buf + threadIdx.x * kBytesPerThread;
        uint32_t cnt = 0;
#pragma unroll
        for (uint32_t i = 0; i < kBytesPerThread; ++i)
            cnt += mine[i] != '\n' ? 1u : 0u;
        uint32_t before = 0;
        Scan(scanTmp).ExclusiveSum(cnt, before);
        // this thread's bases are output bases [o, o + cnt): at most two
        // sequence words (32 bases each) and two mask words (64 each)
        const uint64_t o = tileOut[t] + before;
        const uint64_t sw0 = o >> 5, mw0 = o >> 6;
        unsigned long long s[2] = {0, 0}, m[2] = {0, 0};
        uint32_t j = 0;
#pragma unroll
        for (uint32_t i = 0; i < kBytesPerThread; ++i) {
            const uint8_t b = mine[i];
            if (b == '\n')
                continue;
            const uint64_t pos = o + j++;
            uint32_t c = base_code(b);
            if (c > 3) {
                m[(pos >> 6) - mw0] |= 1ull << (pos & 63);
                c = 0;
            }
            s[(pos >> 5) - sw0] |= (unsigned long long)c << (2 * (pos & 31));
        }
        if (s[0])
            atomicOr(seq + sw0, s[0]);
        if (s[1])
            atomicOr(seq + sw0 + 1, s[1]);
        if (m[0])
            atomicOr(mask + mw0, m[0]);
        if (m[1])
            atomicOr(mask + mw0 + 1, m[1]);
        __syncthreads(); // buf and scanTmp are reused by the next tile
    }
}

// Pinned staging for text uploads, per device, kept for the process: each
// of kWorkers threads owns two slots, a stream and one event per slot.
constexpr uint32_t kWorkers = 8;
constexpr uint64_t kChunk = 16ull << 20;

struct Staging {
    bool ready = false;
    char *slot[kWorkers][2] = {};
    cudaStream_t stream[kWorkers] = {};
    cudaEvent_t free_[kWorkers][2] = {};
};
std::mutex g_stagingMu;
Staging g_staging[16];

// Uploads text[0, n) to dText and returns the header starts in file order:
// 0 and every '>' that follows a '\n'. The caller holds g_stagingMu and has
// made `device` current.
ibs_status upload_text(const char *text, uint64_t n, uint8_t *dText, int device, std::vector<uint64_t> &heads)
{
    Staging &sg = g_staging[device];
    if (!sg.ready) {
        for (uint32_t t = 0; t < kWorkers; ++t) {
            IBS_CUDA(cudaStreamCreateWithFlags(&sg.stream[t], cudaStreamNonBlocking), "stream create");
            for (int i = 0; i < 2; ++i) {
                IBS_CUDA(cudaMallocHost(&sg.slot[t][i], kChunk), "pinned text staging");
                IBS_CUDA(cudaEventCreateWithFlags(&sg.free_[t][i], cudaEventDisableTiming), "event create");
            }
        }
        sg.ready = true;
    }
    const uint64_t nChunks = (n + kChunk - 1) / kChunk;
    const uint32_t nWorkers = (uint32_t)std::min<uint64_t>(kWorkers, nChunks);
    std::vector<std::vector<uint64_t>> found(nChunks);
    std::vector<cudaError_t> err(nWorkers, cudaSuccess);
    auto work = [&](uint32_t t) {
        cudaError_t e = cudaSetDevice(device);
        for (uint64_t c = t, i = 0; c < nChunks && e == cudaSuccess; c += nWorkers, ++i) {
            const uint64_t a = c * kChunk, len = std::min(kChunk, n - a);
            char *slot = sg.slot[t][i & 1];
            e = cudaEventSynchronize(sg.free_[t][i & 1]); // its previous copy has finished
            if (e != cudaSuccess)
                break;
            std::memcpy(slot, text + a, len);
            e = cudaMemcpyAsync(dText + a, slot, len, cudaMemcpyHostToDevice, sg.stream[t]);
            if (e == cudaSuccess)
                e = cudaEventRecord(sg.free_[t][i & 1], sg.stream[t]);
            for (uint64_t q = a; q < a + len;) {
                const char *gt = (const char *)std::memchr(text + q, '>', a + len - q);
                if (!gt)
                    break;
                const uint64_t j = (uint64_t)(gt - text);
                if (j == 0 || text[j - 1] == '\n')
                    found[c].push_back(j);
                q = j + 1;
            }
        }
        if (e == cudaSuccess)
            e = cudaStreamSynchronize(sg.stream[t]);
        err[t] = e;
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nWorkers; ++t)
        pool.emplace_back(work, t);
    if (nWorkers)
        work(0);
    for (auto &th : pool)
        th.join();
    for (cudaError_t e : err)
        if (e != cudaSuccess)
            return cuda_fail(e, "fasta text upload");
    heads.clear();
    for (const auto &f : found)
        heads.insert(heads.end(), f.begin(), f.end());
    return IBS_OK;
}

int grid_for_tiles(uint64_t nTiles)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(nTiles, (uint64_t)sms * 8));
}

} // namespace fasta
} // namespace ibs

using namespace ibs;
using namespace ibs::fasta;

extern "C" ibs_status ibs_reference_from_fasta(const char *text, uint64_t n, int device, ibs_reference **out)
{
    clear_error();
    if (!out || (n && !text)) {
        set_error("ibs_reference_from_fasta: bad argument");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    ibs_status st = check_device_ordinal(device);
    if (st != IBS_OK)
        return st;
    if (device >= 16) {
        set_error("ibs_reference_from_fasta: device ordinal beyond 15");
        return IBS_ERR_ARG;
    }
    if (n == 0) {
        set_error("Empty file");
        return IBS_ERR_FORMAT;
    }
    if (text[0] == '@') {
        set_error("FASTQ text: read it on the host (ibs_pack_ascii)");
        return IBS_ERR_UNSUPPORTED;
    }
    if (text[0] != '>') {
        set_error("Unknown file type");
        return IBS_ERR_FORMAT;
    }
    DeviceGuard guard(device);
    uint8_t *dText = nullptr;
    Tile *dTiles = nullptr;
    uint32_t *dCounts = nullptr;
    uint64_t *dTileOut = nullptr;
    auto freeAll = [&]() {
        cudaFree(dText);
        cudaFree(dTiles);
        cudaFree(dCounts);
        cudaFree(dTileOut);
    };
    struct Guard {
        std::function<void()> f;
        ~Guard() { f(); }
    } g{freeAll};
    IBS_CUDA(cudaMalloc(&dText, n), "fasta text alloc");
    std::vector<uint64_t> heads;
    {
        std::lock_guard<std::mutex> lock(g_stagingMu);
        st = upload_text(text, n, dText, device, heads);
    }
    if (st != IBS_OK)
        return st;
    // records: the id is the rest of the header line, the body runs from the
    // next line up to the next header
    const uint32_t nBodies = (uint32_t)heads.size();
    std::vector<std::string> ids(nBodies);
    std::vector<uint64_t> bodyStart(nBodies), bodyEnd(nBodies);
    for (uint32_t b = 0; b < nBodies; ++b) {
        const uint64_t h = heads[b];
        const uint64_t lim = b + 1 < nBodies ? heads[b + 1] : n;
        const char *nl = (const char *)std::memchr(text + h, '\n', lim - h);
        const uint64_t eol = nl ? (uint64_t)(nl - text) : lim;
        ids[b].assign(text + h + 1, eol - h - 1);
        bodyStart[b] = nl ? eol + 1 : lim;
        bodyEnd[b] = lim;
    }
    std::vector<Tile> tiles;
    for (uint32_t b = 0; b < nBodies; ++b)
        for (uint64_t s = bodyStart[b]; s < bodyEnd[b]; s += kTile)
            tiles.push_back(Tile{s, (uint32_t)std::min<uint64_t>(kTile, bodyEnd[b] - s), b});
    const uint64_t nTiles = tiles.size();
    IBS_CUDA(cudaMalloc(&dTiles, std::max<uint64_t>(nTiles, 1) * sizeof(Tile)), "fasta tiles alloc");
    IBS_CUDA(cudaMalloc(&dCounts, std::max<uint64_t>(nTiles, 1) * 4), "fasta tiles alloc");
    IBS_CUDA(cudaMalloc(&dTileOut, std::max<uint64_t>(nTiles, 1) * 8), "fasta tiles alloc");
    std::vector<uint32_t> counts(nTiles);
    if (nTiles) {
        IBS_CUDA(cudaMemcpy(dTiles, tiles.data(), nTiles * sizeof(Tile), cudaMemcpyHostToDevice),
                 "fasta tiles upload");
        k_count_tiles<<<grid_for_tiles(nTiles), kThreads>>>(dText, dTiles, nTiles, dCounts);
        IBS_LAUNCHED();
        IBS_CUDA(cudaGetLastError(), "fasta count launch");
        IBS_CUDA(cudaMemcpy(counts.data(), dCounts, nTiles * 4, cudaMemcpyDeviceToHost), "fasta counts");
    }
    // records with sequence bytes become contigs, in file order
    std::vector<uint64_t> bodyLen(nBodies, 0);
    for (uint64_t t = 0; t < nTiles; ++t)
        bodyLen[tiles[t].body] += counts[t];
    std::vector<uint64_t> lens;
    std::vector<std::string> keptIds;
    std::vector<int64_t> contigOf(nBodies, -1);
    for (uint32_t b = 0; b < nBodies; ++b)
        if (bodyLen[b]) {
            contigOf[b] = (int64_t)lens.size();
            lens.push_back(bodyLen[b]);
            keptIds.push_back(std::move(ids[b]));
        }
    st = check_contig_lengths(lens.data(), (uint32_t)lens.size(), "ibs_reference_from_fasta");
    if (st != IBS_OK)
        return st;
    std::vector<uint64_t> off;
    uint64_t sw = 0, mw = 0;
    packed_offsets(lens.data(), (uint32_t)lens.size(), off, sw, mw);
    std::vector<uint64_t> tileOut(nTiles);
    {
        std::vector<uint64_t> run(nBodies, 0);
        for (uint64_t t = 0; t < nTiles; ++t) {
            const uint32_t b = tiles[t].body;
            tileOut[t] = contigOf[b] >= 0 ? off[contigOf[b]] + run[b] : 0;
            run[b] += counts[t];
        }
    }
    uint64_t *dSeq = nullptr, *dMask = nullptr;
    cudaError_t e = cudaMalloc(&dSeq, sw * 8);
    if (e == cudaSuccess)
        e = cudaMalloc(&dMask, mw * 8);
    if (e == cudaSuccess)
        e = cudaMemset(dSeq, 0, sw * 8);
    if (e == cudaSuccess)
        e = cudaMemset(dMask, 0, mw * 8);
    if (e == cudaSuccess && nTiles)
        e = cudaMemcpy(dTileOut, tileOut.data(), nTiles * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nTiles) {
        k_pack_tiles<<<grid_for_tiles(nTiles), kThreads>>>(dText, dTiles, nTiles, dTileOut,
                                                           reinterpret_cast<unsigned long long *>(dSeq),
                                                           reinterpret_cast<unsigned long long *>(dMask));
        IBS_LAUNCHED();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(dSeq);
        cudaFree(dMask);
        return cuda_fail(e, "fasta pack");
    }
    ibs_reference *r = nullptr;
    st = reference_adopt(lens, device, dSeq, dMask, &r);
    if (st != IBS_OK)
        return st;
    r->ids = std::move(keptIds);
    *out = r;
    return IBS_OK;
}

extern "C" uint32_t ibs_reference_contig_count(const ibs_reference *r)
{
    return r ? (uint32_t)r->lens.size() : 0;
}

extern "C" ibs_status ibs_reference_contig(const ibs_reference *r, uint32_t i, uint64_t *len, const char **id)
{
    clear_error();
    if (!r || i >= r->lens.size()) {
        set_error("ibs_reference_contig: bad argument");
        return IBS_ERR_ARG;
    }
    if (len)
        *len = r->lens[i];
    if (id)
        *id = i < r->ids.size() ? r->ids[i].c_str() : "";
    return IBS_OK;
}

extern "C" ibs_status ibs_reference_copy_packed(const ibs_reference *r, uint64_t *seq2bit, uint64_t *nmask)
{
    clear_error();
    if (!r || !seq2bit || !nmask) {
        set_error("ibs_reference_copy_packed: bad argument");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(r->device);
    IBS_CUDA(cudaMemcpy(seq2bit, r->dSeq, r->seqWords * 8, cudaMemcpyDeviceToHost), "reference download");
    IBS_CUDA(cudaMemcpy(nmask, r->dMask, r->maskWords * 8, cudaMemcpyDeviceToHost), "reference download");
    return IBS_OK;
}
