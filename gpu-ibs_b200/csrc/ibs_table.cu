// Device table: KMC 3 decode and the sector-bucket build.
//
// ibs_open reads the KMC 3 random-access files with the same layout rules as
// the reference's KmcRaIndex (src/gpu/KmcRaIndex.hpp:497-708): header fields
// and version from the end of .kmc_pre, the bin-major prefix LUT with KMC's
// total+1 guard, and big-endian suffix records followed by counter bytes in
// .kmc_suf. Records are decoded on the device (prefix from the LUT bucket,
// suffix bytes to an integer, counters dropped) straight into canonical
// codes, which the build then hashes into 32-byte buckets.
#include "ibs_internal.cuh"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <unistd.h>

namespace ibs {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_error;

void set_error(const std::string &msg) { g_error = msg; }
void clear_error() { g_error.clear(); }

std::atomic<uint64_t> &launch_counter()
{
    static std::atomic<uint64_t> c{0};
    return c;
}

ibs_status cuda_fail(cudaError_t e, const char *what)
{
    set_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
    cudaGetLastError(); // clear a sticky-free error so the next call starts clean
    return e == cudaErrorMemoryAllocation ? IBS_ERR_NOMEM : IBS_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
static uint32_t floor_log2(uint64_t x) { return 63u - (uint32_t)__builtin_clzll(x); }

static uint64_t next_pow2(uint64_t x)
{
    uint64_t p = 1;
    while (p < x)
        p <<= 1;
    return p;
}

static TableGeom choose_geometry(uint64_t nKeys, uint32_t k, const ibs_table_opts *o)
{
    TableGeom g{};
    g.k = k;
    g.bits = 2 * k;
    uint32_t fmt = o ? o->force_format : 0;
    const bool tunedMz = tuning().table_format == FMT_MZ8;
    // minimum line count of a minimizer table: its slot values must fit 31
    // bits (B8x32 sectors, k <= 27) or 40 bits (B6x40 sectors, k <= 31)
    auto mzMinLog2 = [&](uint32_t f) { return (int)(2 * k) - (f == FMT_MZ8 ? 27 : 36); };
    if (fmt == 0 && tunedMz && k >= 16 && k <= 31) {
        // the tuned default, where the minimizer layout applies and its
        // minimum line count does not oversize the table
        const uint32_t f = k <= 27 ? FMT_MZ8 : FMT_MZ6;
        const double want = (double)nKeys / tuning().keys_per_bucket / mz::kSectorsPerLine;
        if (mzMinLog2(f) <= 0 || want >= (double)(1ull << mzMinLog2(f)))
            fmt = f;
    }
    if (fmt == FMT_AUTO_HASH)
        fmt = 0;
    // the tuned load belongs to the tuned layout; hash tables under a tuned
    // minimizer default keep the hash layout's default of 4 keys per bucket
    double lam = tuning().keys_per_bucket;
    if (tunedMz && !is_mz(fmt))
        lam = 4.0;
    if (o && o->keys_per_bucket > 0)
        lam = o->keys_per_bucket;
    const uint64_t space = g.bits >= 64 ? ~0ull : (1ull << g.bits);
    auto clampN = [&](uint64_t n) {
        if (n < 1)
            n = 1;
        if (g.bits < 64 && n > space)
            n = space;
        return n;
    };
    const uint64_t n8 = clampN((uint64_t)((double)nKeys / lam) + 1);
    const uint64_t min8 = g.bits > 31 ? (1ull << (g.bits - 31)) : 1;
    const uint64_t n6 = clampN((uint64_t)((double)nKeys / (lam * 6.0 / 8.0)) + 1);
    const uint64_t min6 = g.bits > 40 ? (1ull << (g.bits - 40)) : 1;
    if (is_mz(fmt)) {
        // minimizer lines of four sectors, at least 2^mzMinLog2 of them
        g.format = fmt;
        const uint32_t m = mz::m_of(k);
        const uint64_t minLines = mzMinLog2(fmt) > 0 ? (1ull << mzMinLog2(fmt)) : 1;
        const uint64_t want = fmt == FMT_MZ8 ? n8 : n6; // sectors at the load
        const uint64_t nLines =
            std::min<uint64_t>(std::max((want + mz::kSectorsPerLine - 1) / mz::kSectorsPerLine, minLines),
                               1ull << 31); // line_of needs nLines < 2^32
        g.nBuckets = nLines * mz::kSectorsPerLine;
        g.fpBits = 2 * m - floor_log2(nLines);
        g.stashBuckets = 0;
        return g;
    }
    if (fmt == 0)
        fmt = (std::max(n8, min8) <= 2 * n8) ? FMT_B8X32 : FMT_B6X40;
    g.format = fmt;
    g.nBuckets = fmt == FMT_B8X32 ? std::max(n8, min8) : std::max(n6, min6);
    g.nBuckets = clampN(g.nBuckets);
    int fpb = (int)g.bits - (int)floor_log2(g.nBuckets);
    g.fpBits = (uint32_t)std::max(fpb, 1);
    g.stashBuckets = 0;
    return g;
}

// ---------------------------------------------------------------------------
// build kernels
// ---------------------------------------------------------------------------
// Bucket and stored fingerprint of a key in either table family.
__device__ __forceinline__ void locate_key(uint64_t code, const TableGeom &g, uint64_t &r, uint64_t &fp)
{
    if (is_mz(g.format)) {
        mz::locate(code, g, r, fp);
        return;
    }
    const uint64_t h = perm_hash(code, g.bits);
    r = bucket_of(h, g);
    fp = fp_of(h, g);
}

__global__ void k_count(const uint64_t *__restrict__ codes, uint64_t n, TableGeom g,
                        uint32_t *__restrict__ cnt)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r, fp;
        locate_key(codes[i], g, r, fp);
        atomicAdd(cnt + r, 1u);
    }
}

// Marks overflowing buckets, records B6x40 counts, sums the keys that go to
// the stash and resets the counters for the placement pass.
__global__ void k_mark(uint32_t *__restrict__ cnt, uint64_t nb, TableGeom g,
                       uint32_t *__restrict__ words, unsigned long long *__restrict__ overflowKeys)
{
    unsigned long long local = 0;
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < nb;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = cnt[r];
        if (g.format == FMT_B8X32) {
            if (c > 8) {
                words[r * 8 + 7] = B8_OVERFLOW;
                local += c - 7;
            }
        } else {
            const uint32_t keep = c > 6 ? 6 : c;
            const uint32_t flags = c > 6 ? 1u : 0u;
            if (c > 6)
                local += c - 6;
            words[r * 8 + 7] = (words[r * 8 + 7] & 0x0000ffffu) | (keep << 16) | (flags << 24);
        }
        cnt[r] = 0;
    }
    for (int o = 16; o; o >>= 1)
        local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local)
        atomicAdd(overflowKeys, local);
}

// MZ8: marks full sectors pair by pair (sectors 2i and 2i + 1 of a line are
// partners). A sector with c > 8 keys keeps 7 and sends c - 7 to its
// partner's free slots (8 - c' when the partner holds c' < 8) and the rest to
// the stash. Sums the keys leaving their sector (spill) and those reaching
// the stash, and resets the counters for the placement pass.
__global__ void k_mark_mz8(uint32_t *__restrict__ cnt, uint64_t nb, uint32_t *__restrict__ words,
                           unsigned long long *__restrict__ spillKeys, unsigned long long *__restrict__ stashKeys)
{
    unsigned long long spill = 0, stash = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; 2 * i < nb;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = 2 * i;
        const uint32_t c[2] = {cnt[r], cnt[r + 1]};
        for (int a = 0; a < 2; ++a) {
            if (c[a] > 8) {
                const uint32_t extra = c[a] - 7;
                const uint32_t room = c[a ^ 1] < 8 ? 8 - c[a ^ 1] : 0;
                words[(r + a) * 8 + 7] = extra > room ? B8_OVERFLOW_STASH : B8_OVERFLOW;
                spill += extra;
                stash += extra > room ? extra - room : 0;
            }
        }
        cnt[r] = cnt[r + 1] = 0;
    }
    for (int o = 16; o; o >>= 1) {
        spill += __shfl_xor_sync(0xffffffffu, spill, o);
        stash += __shfl_xor_sync(0xffffffffu, stash, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (spill)
            atomicAdd(spillKeys, spill);
        if (stash)
            atomicAdd(stashKeys, stash);
    }
}

__device__ __forceinline__ bool stash_insert(uint64_t *stash, uint64_t stashBuckets, uint64_t code)
{
    uint64_t b = stash_home(code, stashBuckets);
    for (uint64_t i = 0; i < stashBuckets; ++i) {
        for (int s = 0; s < 4; ++s) {
            unsigned long long *slot = reinterpret_cast<unsigned long long *>(stash + 4 * b + s);
            const unsigned long long old = atomicCAS(slot, (unsigned long long)STASH_EMPTY,
                                                     (unsigned long long)code);
            if (old == STASH_EMPTY || old == code)
                return true;
        }
        b = (b + 1) & (stashBuckets - 1);
    }
    return false;
}

// Places every key in its bucket; the extra keys of a full bucket go to the
// stash, or for MZ8 to the spill list (placed by k_spill_mz8 once every
// sector holds its own keys).
__global__ void k_place(const uint64_t *__restrict__ codes, uint64_t n, TableGeom g,
                        uint32_t *__restrict__ cnt, uint32_t *__restrict__ words,
                        uint64_t *__restrict__ stash, uint64_t *__restrict__ spillList,
                        unsigned long long *__restrict__ spillN, uint64_t spillCap, int *__restrict__ err)
{
    uint8_t *bytes = reinterpret_cast<uint8_t *>(words);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t code = codes[i];
        uint64_t r, fp;
        locate_key(code, g, r, fp);
        const uint32_t s = atomicAdd(cnt + r, 1u);
        bool stashed = false;
        if (g.format == FMT_MZ8) {
            const uint32_t w7 = words[r * 8 + 7];
            const uint32_t limit = (w7 == B8_OVERFLOW || w7 == B8_OVERFLOW_STASH) ? 7u : 8u;
            if (s < limit) {
                words[r * 8 + s] = (uint32_t)fp;
            } else {
                const unsigned long long j = atomicAdd(spillN, 1ull);
                if (j < spillCap)
                    spillList[j] = code;
                else
                    atomicExch(err, 1);
            }
        } else if (g.format == FMT_B8X32) {
            const uint32_t limit = words[r * 8 + 7] == B8_OVERFLOW ? 7u : 8u;
            if (s < limit)
                words[r * 8 + s] = (uint32_t)fp;
            else
                stashed = true;
        } else {
            if (s < 6) {
                words[r * 8 + s] = (uint32_t)(fp >> 8);
                bytes[r * 32 + 24 + s] = (uint8_t)(fp & 0xff);
            } else
                stashed = true;
        }
        if (stashed && !stash_insert(stash, g.stashBuckets, code))
            atomicExch(err, 1);
    }
}

// MZ8 spill pass: each extra key takes the next free slot of its partner
// sector (after the partner's own keys, all placed by k_place), or the stash
// once the partner is full. The numbers that land in each place follow from
// the counts, as k_mark_mz8 recorded them in the sector markers.
__global__ void k_spill_mz8(const uint64_t *__restrict__ spillList, uint64_t n, TableGeom g,
                            uint32_t *__restrict__ cnt, uint32_t *__restrict__ words, uint64_t *__restrict__ stash,
                            int *__restrict__ err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t code = spillList[i];
        uint64_t r, fp;
        locate_key(code, g, r, fp);
        const uint32_t s = atomicAdd(cnt + (r ^ 1), 1u);
        if (s < 8)
            words[(r ^ 1) * 8 + s] = (uint32_t)fp;
        else if (!stash_insert(stash, g.stashBuckets, code))
            atomicExch(err, 1);
    }
}

// Record r of a .kmc_suf chunk -> canonical code. The LUT bucket j holding
// record r is the last j with lut[j] <= r (empty buckets repeat a value and
// are skipped by taking the last); j mod 4^p is the prefix.
__global__ void k_decode(const uint8_t *__restrict__ raw, uint64_t r0, uint64_t nRec,
                         uint32_t recBytes, uint32_t sufBytes, const uint64_t *__restrict__ lut,
                         uint64_t lutN, uint64_t prefixMask, uint32_t sufBits,
                         uint64_t *__restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nRec;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = r0 + i;
        uint64_t lo = 0, hi = lutN - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi + 1) >> 1;
            if (__ldg(lut + mid) <= r)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint8_t *q = raw + i * recBytes;
        uint64_t suf = 0;
        for (uint32_t b = 0; b < sufBytes; ++b)
            suf = (suf << 8) | q[b];
        const uint64_t prefix = lo & prefixMask;
        out[r] = sufBits >= 64 ? suf : ((prefix << sufBits) | suf);
    }
}

// The same for 33 <= k <= 64: the suffix (up to 16 bytes) and the prefix
// shifted above it as a 128-bit code {lo, hi}; sufBits = 2 (k - p) > 0.
__global__ void k_decode_wide(const uint8_t *__restrict__ raw, uint64_t r0, uint64_t nRec, uint32_t recBytes,
                              uint32_t sufBytes, const uint64_t *__restrict__ lut, uint64_t lutN,
                              uint64_t prefixMask, uint32_t sufBits, ulonglong2 *__restrict__ out)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nRec;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = r0 + i;
        uint64_t lo = 0, hi = lutN - 1;
        while (lo < hi) {
            const uint64_t mid = (lo + hi + 1) >> 1;
            if (__ldg(lut + mid) <= r)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint8_t *q = raw + i * recBytes;
        uint64_t slo = 0, shi = 0;
        for (uint32_t b = 0; b < sufBytes; ++b) {
            shi = (shi << 8) | (slo >> 56);
            slo = (slo << 8) | q[b];
        }
        const uint64_t prefix = lo & prefixMask;
        if (sufBits >= 64) {
            shi |= prefix << (sufBits - 64);
        } else {
            slo |= prefix << sufBits;
            shi |= prefix >> (64 - sufBits);
        }
        out[r] = make_ulonglong2(slo, shi);
    }
}

template <uint32_t FMT>
__global__ void k_probe(TableView t, const uint64_t *__restrict__ codes, uint64_t n,
                        uint8_t *__restrict__ hits)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        hits[i] = table_lookup<FMT>(t, codes[i]) ? 1 : 0;
}

// Number of codes present in the table: each thread counts its share, each
// warp adds its lanes' counts and one lane adds the warp's to the total.
template <uint32_t FMT>
__global__ void k_count_present(TableView t, const uint64_t *__restrict__ codes, uint64_t n,
                                unsigned long long *__restrict__ count)
{
    unsigned long long local = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        local += table_lookup<FMT>(t, codes[i]) ? 1 : 0;
    for (int o = 16; o; o >>= 1)
        local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local)
        atomicAdd(count, local);
}

static int grid_for(uint64_t n, int threads)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * 16;
    return (int)std::max<uint64_t>(1, std::min(want, cap));
}

// Builds the table from device codes. The caller has set the device.
static ibs_status build_from_device_codes(ibs_table *t, const uint64_t *dCodes, uint64_t n,
                                          uint32_t k, const ibs_table_opts *o)
{
    t->geom = choose_geometry(n, k, o);
    t->nKeys = n;
    TableGeom &g = t->geom;
    const uint64_t nb = g.nBuckets;
    IBS_CUDA(cudaMalloc(&t->buckets, nb * 32), "table alloc");
    t->deviceBytes = nb * 32;
    IBS_CUDA(cudaMemset(t->buckets, g.format == FMT_B6X40 || g.format == FMT_MZ6 ? 0x00 : 0xff, nb * 32),
             "table init");
    uint32_t *cnt = nullptr;
    unsigned long long *dOverflow = nullptr; // [0] keys to the stash, [1] MZ8 spill keys, [2] spill list fill
    uint64_t *spillList = nullptr;
    int *dErr = nullptr;
    auto cleanup = [&]() {
        cudaFree(cnt);
        cudaFree(dOverflow);
        cudaFree(spillList);
        cudaFree(dErr);
    };
    cudaError_t e = cudaMalloc(&cnt, nb * 4);
    if (e == cudaSuccess)
        e = cudaMalloc(&dOverflow, 3 * 8);
    if (e == cudaSuccess)
        e = cudaMalloc(&dErr, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemset(cnt, 0, nb * 4);
    if (e == cudaSuccess)
        e = cudaMemset(dOverflow, 0, 3 * 8);
    if (e == cudaSuccess)
        e = cudaMemset(dErr, 0, sizeof(int));
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "table build scratch");
    }
    uint32_t *words = reinterpret_cast<uint32_t *>(t->buckets);
    k_count<<<grid_for(n, 256), 256>>>(dCodes, n, g, cnt);
    IBS_LAUNCHED();
    if (g.format == FMT_MZ8)
        k_mark_mz8<<<grid_for(nb / 2, 256), 256>>>(cnt, nb, words, dOverflow + 1, dOverflow);
    else
        k_mark<<<grid_for(nb, 256), 256>>>(cnt, nb, g, words, dOverflow);
    IBS_LAUNCHED();
    unsigned long long counts[2] = {0, 0}; // keys to the stash, MZ8 keys leaving their sector
    e = cudaMemcpy(counts, dOverflow, 2 * 8, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && counts[1])
        e = cudaMalloc(&spillList, counts[1] * 8);
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "table build count");
    }
    const unsigned long long overflow = counts[0];
    t->stashKeys = overflow;
    if (overflow) {
        g.stashBuckets = next_pow2((overflow * 2 + 3) / 4);
        e = cudaMalloc(&t->stash, g.stashBuckets * 32);
        if (e == cudaSuccess)
            e = cudaMemset(t->stash, 0xff, g.stashBuckets * 32);
        if (e != cudaSuccess) {
            cleanup();
            return cuda_fail(e, "stash alloc");
        }
        t->deviceBytes += g.stashBuckets * 32;
    }
    k_place<<<grid_for(n, 256), 256>>>(dCodes, n, g, cnt, words, t->stash, spillList, dOverflow + 2, counts[1],
                                       dErr);
    IBS_LAUNCHED();
    if (counts[1]) {
        k_spill_mz8<<<grid_for(counts[1], 256), 256>>>(spillList, counts[1], g, cnt, words, t->stash, dErr);
        IBS_LAUNCHED();
    }
    int herr = 0;
    e = cudaMemcpy(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost);
    cleanup();
    if (e != cudaSuccess)
        return cuda_fail(e, "table build place");
    if (herr) {
        set_error("table build: stash full");
        return IBS_ERR_CAPACITY;
    }
    return IBS_OK;
}

// ---------------------------------------------------------------------------
// KMC 3 files (layout as read by src/gpu/KmcRaIndex.hpp:497-708)
// ---------------------------------------------------------------------------
struct KmcHeader {
    uint32_t version = 0, k = 0, mode = 0, counterSize = 0, p = 0, sigLen = 0;
    uint64_t total = 0, headerOffset = 0, fileBytes = 0;
};

struct File {
    FILE *f = nullptr;
    explicit File(const std::string &path) { f = fopen(path.c_str(), "rb"); }
    ~File()
    {
        if (f)
            fclose(f);
    }
};

static bool read_at(FILE *f, long long off, void *dst, size_t n)
{
    if (fseeko(f, off, SEEK_SET) != 0)
        return false;
    return fread(dst, 1, n, f) == n;
}

static uint64_t file_size(FILE *f)
{
    fseeko(f, 0, SEEK_END);
    return (uint64_t)ftello(f);
}

static ibs_status check_markers(FILE *f, uint64_t size, const char *marker, const std::string &path)
{
    char head[4], tail[4];
    if (size < 8 || !read_at(f, 0, head, 4) || !read_at(f, (long long)size - 4, tail, 4)) {
        set_error("KMC: short read of markers in " + path);
        return IBS_ERR_IO;
    }
    if (memcmp(head, marker, 4) || memcmp(tail, marker, 4)) {
        set_error("KMC: bad marker in " + path);
        return IBS_ERR_FORMAT;
    }
    return IBS_OK;
}

// maxK: 32 for the callers that take one-word codes, 64 for those that also
// take wide-key codes.
static ibs_status read_kmc_header(FILE *f, const std::string &path, KmcHeader &h, uint32_t maxK = 32)
{
    h.fileBytes = file_size(f);
    ibs_status s = check_markers(f, h.fileBytes, "KMCP", path);
    if (s != IBS_OK)
        return s;
    if (h.fileBytes < 20 || !read_at(f, (long long)h.fileBytes - 12, &h.version, 4)) {
        set_error("KMC: short read of version in " + path);
        return IBS_ERR_IO;
    }
    if (h.version != 0 && h.version != 0x200) {
        set_error("KMC: unsupported KMC format version in " + path);
        return IBS_ERR_FORMAT;
    }
    unsigned char off = 0; // only the first byte of header_offset is read, as KMC does
    if (!read_at(f, (long long)h.fileBytes - 8, &off, 1)) {
        set_error("KMC: short read of header offset in " + path);
        return IBS_ERR_IO;
    }
    h.headerOffset = off;
    const long long pos = (long long)h.fileBytes - (long long)(h.headerOffset + 8);
    if (pos < 4) {
        set_error("KMC: header offset out of range in " + path);
        return IBS_ERR_FORMAT;
    }
    if (h.version == 0x200) {
        uint32_t w[5];
        if (!read_at(f, pos, w, sizeof w) || !read_at(f, pos + 28, &h.total, 8)) {
            set_error("KMC: short read of header in " + path);
            return IBS_ERR_IO;
        }
        h.k = w[0], h.mode = w[1], h.counterSize = w[2], h.p = w[3], h.sigLen = w[4];
    } else {
        uint32_t w[4];
        if (!read_at(f, pos, w, sizeof w) || !read_at(f, pos + 24, &h.total, 8)) {
            set_error("KMC: short read of header in " + path);
            return IBS_ERR_IO;
        }
        h.k = w[0], h.mode = w[1], h.counterSize = w[2], h.p = w[3];
    }
    if (h.mode != 0) {
        set_error("KMC: Quake-compatible counters are not supported");
        return IBS_ERR_UNSUPPORTED;
    }
    if (h.k == 0 || h.k > maxK) {
        set_error("KMC: k=" + std::to_string(h.k) + " is not supported (k must be 1.." + std::to_string(maxK) +
                  (maxK < kMaxWideK ? " here; wide-key tables take k up to 64)" : ")"));
        return IBS_ERR_UNSUPPORTED;
    }
    if (h.p > h.k || (h.k - h.p) % 4 != 0 || h.k - h.p > maxK || h.p > 31) {
        set_error("KMC: unexpected suffix geometry");
        return IBS_ERR_FORMAT;
    }
    return IBS_OK;
}

// Reads the prefix LUT (bin-major for 0x200) with the guard set to
// total + 1 as KMC sets it (src/gpu/KmcRaIndex.hpp:564-591).
static ibs_status read_kmc_lut(FILE *f, const std::string &path, const KmcHeader &h,
                               std::vector<uint64_t> &lut)
{
    uint64_t entries;
    if (h.version == 0x200) {
        const uint64_t sigEntries = (1ull << (2 * h.sigLen)) + 1;
        const uint64_t fixed = sigEntries * 4 + h.headerOffset + 8 + 12;
        if (h.fileBytes < fixed) {
            set_error("KMC: .kmc_pre too small in " + path);
            return IBS_ERR_FORMAT;
        }
        const uint64_t lutArea = h.fileBytes - 12 - (sigEntries * 4 + h.headerOffset + 8);
        entries = (lutArea + 8) / 8;
    } else {
        entries = (1ull << (2 * h.p)) + 1;
    }
    const uint64_t single = 1ull << (2 * h.p);
    if (entries < 2 || (entries - 1) % single != 0) {
        set_error("KMC: LUT size is not a whole number of bins in " + path);
        return IBS_ERR_FORMAT;
    }
    lut.resize(entries);
    if (!read_at(f, 4, lut.data(), entries * 8)) {
        set_error("KMC: short read of prefix LUT in " + path);
        return IBS_ERR_IO;
    }
    lut[entries - 1] = h.total + 1;
    return IBS_OK;
}

} // namespace ibs

using namespace ibs;

// ---------------------------------------------------------------------------
// C-ABI
// ---------------------------------------------------------------------------
extern "C" const char *ibs_last_error(void) { return ibs::g_error.c_str(); }

extern "C" int ibs_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

extern "C" uint64_t ibs_launch_count(void) { return launch_counter().load(); }


static ibs_status check_format(uint32_t k, const ibs_table_opts *o)
{
    if (o && o->force_format == FMT_WIDE && k <= 32) {
        set_error("wide-key tables (format 8) need 33 <= k <= 64");
        return IBS_ERR_UNSUPPORTED;
    }
    if (k > 32) {
        if (o && o->force_format && o->force_format != FMT_WIDE) {
            set_error("k=" + std::to_string(k) + " > 32 takes only the wide-key table layout (format 8)");
            return IBS_ERR_UNSUPPORTED;
        }
        return IBS_OK;
    }
    if (o && o->force_format == FMT_MZ8 && (k < 16 || k > 27)) {
        set_error("minimizer-bucketed tables (format 4) need 16 <= k <= 27");
        return IBS_ERR_UNSUPPORTED;
    }
    if (o && o->force_format == FMT_MZ6 && (k < 16 || k > 31)) {
        set_error("minimizer-bucketed tables with 40-bit slots (format 6) need 16 <= k <= 31");
        return IBS_ERR_UNSUPPORTED;
    }
    if (o && ((o->force_format > FMT_MZ6 && o->force_format != FMT_WIDE) || o->force_format == FMT_PANEL)) {
        set_error("unknown table format " + std::to_string(o->force_format));
        return IBS_ERR_ARG;
    }
    return IBS_OK;
}

extern "C" ibs_status ibs_table_from_codes(const uint64_t *codes, uint64_t n, uint32_t k,
                                           int codes_on_device, const ibs_table_opts *opts,
                                           ibs_table **out)
{
    clear_error();
    if (!out || (!codes && n) || k == 0 || k > 32) {
        set_error(k > 32 ? "ibs_table_from_codes: k > 32 codes take two words (ibs_table_from_codes128)"
                         : "ibs_table_from_codes: bad argument");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    const int dev = opts ? opts->device : 0;
    ibs_status s = check_format(k, opts);
    if (s != IBS_OK)
        return s;
    s = check_device_ordinal(dev);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(dev);
    const auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<ibs_table> t(new ibs_table);
    t->device = dev;
    uint64_t *dCodes = nullptr;
    const uint64_t *src = codes;
    if (!codes_on_device && n) {
        IBS_CUDA(cudaMalloc(&dCodes, n * 8), "codes alloc");
        cudaError_t e = cudaMemcpy(dCodes, codes, n * 8, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(dCodes);
            return cuda_fail(e, "codes upload");
        }
        src = dCodes;
    }
    s = build_from_device_codes(t.get(), src, n, k, opts);
    cudaFree(dCodes);
    if (s != IBS_OK) {
        ibs_close(t.release());
        return s;
    }
    t->buildSeconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = t.release();
    return IBS_OK;
}

ibs_status ibs::check_device_ordinal(int dev)
{
    const int n = ibs_device_count();
    if (n == 0) {
        set_error("no usable CUDA device (the scan has no CPU fallback)");
        return IBS_ERR_CUDA;
    }
    if (dev < 0 || dev >= n) {
        set_error("device " + std::to_string(dev) + " out of range");
        return IBS_ERR_ARG;
    }
    return IBS_OK;
}

namespace ibs {
// Decodes <prefix>.kmc_pre/.kmc_suf into canonical codes in device memory
// (cudaMalloc'd; the caller frees *dCodes): one word per code for k <= 32,
// {lo, hi} for 33 <= k <= maxK. The device must be current.
static ibs_status decode_kmc_impl(const char *prefix, int dev, uint64_t **dCodesOut, uint64_t *nOut,
                                  uint32_t *kOut, uint32_t maxK)
{
    *dCodesOut = nullptr;
    const std::string pre = std::string(prefix) + ".kmc_pre";
    const std::string suf = std::string(prefix) + ".kmc_suf";
    KmcHeader h;
    std::vector<uint64_t> lut;
    {
        File f(pre);
        if (!f.f) {
            set_error("KMC: cannot open " + pre);
            return IBS_ERR_IO;
        }
        ibs_status s = read_kmc_header(f.f, pre, h, maxK);
        if (s != IBS_OK)
            return s;
        s = read_kmc_lut(f.f, pre, h, lut);
        if (s != IBS_OK)
            return s;
    }
    File sf(suf);
    if (!sf.f) {
        set_error("KMC: cannot open " + suf);
        return IBS_ERR_IO;
    }
    const uint64_t sufSize = file_size(sf.f);
    {
        ibs_status s = check_markers(sf.f, sufSize, "KMCS", suf);
        if (s != IBS_OK)
            return s;
    }
    const uint32_t sufBytes = (h.k - h.p) / 4;
    const uint32_t recBytes = sufBytes + h.counterSize;
    if (recBytes == 0 || sufSize - 8 < h.total * (uint64_t)recBytes) {
        set_error("KMC: suffix file smaller than expected: " + suf);
        return IBS_ERR_FORMAT;
    }
    ibs_status s = check_device_ordinal(dev);
    if (s != IBS_OK)
        return s;
    // The records go up in chunks through a ring of kSlots pinned buffers:
    // kReaders host threads read chunks ahead (pread, in parallel), and this
    // thread uploads and decodes them in order; a buffer is read into again
    // once the upload of its previous chunk has finished.
    constexpr int kSlots = 8, kReaders = 4;
    uint64_t *dCodes = nullptr, *dLut = nullptr;
    uint8_t *dRaw[kSlots] = {};
    uint8_t *hRaw[kSlots] = {};
    cudaEvent_t done[kSlots] = {};
    cudaStream_t st = nullptr;
    const uint64_t total = h.total;
    const uint64_t chunkRecs = std::max<uint64_t>(1, (128ull << 20) / recBytes);
    const uint64_t chunkBytes = chunkRecs * recBytes;
    const uint64_t nChunks = (total + chunkRecs - 1) / chunkRecs;
    const int nSlots = (int)std::min<uint64_t>(kSlots, std::max<uint64_t>(nChunks, 1));
    // ring state: chunk filled[i] is in slot i ready for upload; consumed[i]
    // is the last chunk whose upload from slot i was enqueued
    std::mutex mu;
    std::condition_variable cv;
    std::vector<int64_t> filled(nSlots, -1), consumed(nSlots, -1);
    bool readFailed = false, stopReading = false;
    std::vector<std::thread> readers;
    auto cleanup = [&]() {
        {
            std::lock_guard<std::mutex> lock(mu);
            stopReading = true;
        }
        cv.notify_all();
        for (auto &t : readers)
            t.join();
        readers.clear();
        if (st)
            cudaStreamSynchronize(st);
        cudaFree(dCodes);
        cudaFree(dLut);
        for (int i = 0; i < nSlots; i++) {
            cudaFree(dRaw[i]);
            cudaFreeHost(hRaw[i]);
            if (done[i])
                cudaEventDestroy(done[i]);
        }
        if (st)
            cudaStreamDestroy(st);
    };
    const uint32_t codeWords = h.k > 32 ? 2 : 1;
    cudaError_t e = cudaMalloc(&dCodes, std::max<uint64_t>(total, 1) * 8 * codeWords);
    if (e == cudaSuccess)
        e = cudaMalloc(&dLut, lut.size() * 8);
    if (e == cudaSuccess)
        e = cudaMemcpy(dLut, lut.data(), lut.size() * 8, cudaMemcpyHostToDevice);
    for (int i = 0; i < nSlots && e == cudaSuccess; i++) {
        e = cudaMalloc(&dRaw[i], chunkBytes);
        if (e == cudaSuccess)
            e = cudaMallocHost(&hRaw[i], chunkBytes);
        if (e == cudaSuccess)
            e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "KMC decode buffers");
    }
    const int fd = fileno(sf.f);
    int device = 0;
    cudaGetDevice(&device);
    auto reader = [&](int r) {
        cudaSetDevice(device);
        for (uint64_t c = r; c < nChunks; c += kReaders) {
            const int slot = (int)(c % nSlots);
            {
                // the slot's previous chunk (c - nSlots) must have been enqueued
                std::unique_lock<std::mutex> lock(mu);
                cv.wait(lock, [&] {
                    return stopReading || (c < (uint64_t)nSlots ? true : consumed[slot] == (int64_t)(c - nSlots));
                });
                if (stopReading)
                    return;
            }
            if (c >= (uint64_t)nSlots && cudaEventSynchronize(done[slot]) != cudaSuccess) {
                std::lock_guard<std::mutex> lock(mu);
                readFailed = true;
                cv.notify_all();
                return;
            }
            const uint64_t r0 = c * chunkRecs;
            const uint64_t bytes = std::min(chunkRecs, total - r0) * recBytes;
            uint64_t got = 0;
            while (got < bytes) {
                const ssize_t n = pread(fd, hRaw[slot] + got, bytes - got, (off_t)(4 + r0 * recBytes + got));
                if (n <= 0)
                    break;
                got += (uint64_t)n;
            }
            std::lock_guard<std::mutex> lock(mu);
            if (got != bytes)
                readFailed = true;
            else
                filled[slot] = (int64_t)c;
            cv.notify_all();
            if (got != bytes)
                return;
        }
    };
    for (int r = 0; r < kReaders && (uint64_t)r < nChunks; ++r)
        readers.emplace_back(reader, r);
    const uint64_t lutN = lut.size() - 1;
    const uint64_t prefixMask = (1ull << (2 * h.p)) - 1;
    for (uint64_t c = 0; c < nChunks && e == cudaSuccess; ++c) {
        const int slot = (int)(c % nSlots);
        {
            std::unique_lock<std::mutex> lock(mu);
            cv.wait(lock, [&] { return readFailed || filled[slot] == (int64_t)c; });
            if (readFailed) {
                lock.unlock();
                cleanup();
                set_error("KMC: short read of suffix records in " + suf);
                return IBS_ERR_IO;
            }
        }
        const uint64_t r0 = c * chunkRecs;
        const uint64_t nRec = std::min(chunkRecs, total - r0);
        e = cudaMemcpyAsync(dRaw[slot], hRaw[slot], nRec * recBytes, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess)
            break;
        if (codeWords == 2)
            k_decode_wide<<<grid_for(nRec, 256), 256, 0, st>>>(dRaw[slot], r0, nRec, recBytes, sufBytes, dLut, lutN,
                                                               prefixMask, 2 * (h.k - h.p),
                                                               reinterpret_cast<ulonglong2 *>(dCodes));
        else
            k_decode<<<grid_for(nRec, 256), 256, 0, st>>>(dRaw[slot], r0, nRec, recBytes, sufBytes, dLut, lutN,
                                                          prefixMask, 2 * (h.k - h.p), dCodes);
        IBS_LAUNCHED();
        e = cudaEventRecord(done[slot], st);
        {
            std::lock_guard<std::mutex> lock(mu);
            consumed[slot] = (int64_t)c;
        }
        cv.notify_all();
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess) {
        cleanup();
        return cuda_fail(e, "KMC decode");
    }
    *dCodesOut = dCodes;
    dCodes = nullptr;
    *nOut = total;
    *kOut = h.k;
    cleanup();
    return IBS_OK;
}

ibs_status decode_kmc(const char *prefix, int dev, uint64_t **dCodes, uint64_t *n, uint32_t *k)
{
    return decode_kmc_impl(prefix, dev, dCodes, n, k, 32);
}

ibs_status decode_kmc_any(const char *prefix, int dev, uint64_t **dCodes, uint64_t *n, uint32_t *k)
{
    return decode_kmc_impl(prefix, dev, dCodes, n, k, kMaxWideK);
}
} // namespace ibs

extern "C" ibs_status ibs_open(const char *prefix, const ibs_table_opts *opts, ibs_table **out)
{
    clear_error();
    if (!prefix || !out) {
        set_error("ibs_open: bad argument");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    const int dev = opts ? opts->device : 0;
    {
        // read the header first so a bad file is reported before any device check
        KmcHeader h;
        File f(std::string(prefix) + ".kmc_pre");
        if (!f.f) {
            set_error(std::string("KMC: cannot open ") + prefix + ".kmc_pre");
            return IBS_ERR_IO;
        }
        ibs_status s = read_kmc_header(f.f, std::string(prefix) + ".kmc_pre", h, kMaxWideK);
        if (s != IBS_OK)
            return s;
        s = check_format(h.k, opts);
        if (s != IBS_OK)
            return s;
    }
    ibs_status s = check_device_ordinal(dev);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(dev);
    uint64_t *dCodes = nullptr, total = 0;
    uint32_t k = 0;
    s = decode_kmc_any(prefix, dev, &dCodes, &total, &k);
    if (s != IBS_OK)
        return s;
    std::unique_ptr<ibs_table> t(new ibs_table);
    t->device = dev;
    if (k > 32)
        s = build_wide(t.get(), reinterpret_cast<const ulonglong2 *>(dCodes), total, k, opts);
    else
        s = build_from_device_codes(t.get(), dCodes, total, k, opts);
    cudaFree(dCodes);
    if (s != IBS_OK) {
        ibs_close(t.release());
        return s;
    }
    t->buildSeconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = t.release();
    return IBS_OK;
}

extern "C" ibs_status ibs_table_info_get(const ibs_table *t, ibs_table_info *info)
{
    clear_error();
    if (!t || !info) {
        set_error("ibs_table_info_get: bad argument");
        return IBS_ERR_ARG;
    }
    memset(info, 0, sizeof *info);
    info->k = t->geom.k;
    info->format = t->geom.format;
    info->fp_bits = t->geom.fpBits;
    info->n_keys = t->nKeys;
    info->n_buckets = t->geom.nBuckets;
    info->stash_keys = t->stashKeys;
    info->stash_buckets = t->geom.stashBuckets;
    info->device_bytes = t->deviceBytes;
    info->build_seconds = t->buildSeconds;
    return IBS_OK;
}

extern "C" ibs_status ibs_probe(ibs_table *t, const uint64_t *codes, uint64_t n, uint8_t *hits)
{
    clear_error();
    if (!t || (n && (!codes || !hits))) {
        set_error("ibs_probe: bad argument");
        return IBS_ERR_ARG;
    }
    if (t->geom.format == FMT_WIDE) {
        set_error("ibs_probe: a wide-key table (k > 32) takes ibs_probe128");
        return IBS_ERR_ARG;
    }
    if (!n)
        return IBS_OK;
    DeviceGuard guard(t->device);
    uint64_t *dCodes = nullptr;
    uint8_t *dHits = nullptr;
    cudaError_t e = cudaMalloc(&dCodes, n * 8);
    if (e == cudaSuccess)
        e = cudaMalloc(&dHits, n);
    if (e == cudaSuccess)
        e = cudaMemcpy(dCodes, codes, n * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        if (t->geom.format == FMT_B8X32)
            k_probe<FMT_B8X32><<<grid_for(n, 256), 256>>>(t->view(), dCodes, n, dHits);
        else if (t->geom.format == FMT_MZ8)
            k_probe<FMT_MZ8><<<grid_for(n, 256), 256>>>(t->view(), dCodes, n, dHits);
        else if (t->geom.format == FMT_MZ6)
            k_probe<FMT_MZ6><<<grid_for(n, 256), 256>>>(t->view(), dCodes, n, dHits);
        else
            k_probe<FMT_B6X40><<<grid_for(n, 256), 256>>>(t->view(), dCodes, n, dHits);
        IBS_LAUNCHED();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(hits, dHits, n, cudaMemcpyDeviceToHost);
    cudaFree(dCodes);
    cudaFree(dHits);
    if (e != cudaSuccess)
        return cuda_fail(e, "probe");
    return IBS_OK;
}

// Codes on the device -> how many the table holds.
static ibs_status count_present_device(ibs_table *t, const uint64_t *dCodes, uint64_t n, uint64_t *count)
{
    *count = 0;
    if (!n)
        return IBS_OK;
    unsigned long long *dCount = nullptr;
    IBS_CUDA(cudaMalloc(&dCount, sizeof *dCount), "count alloc");
    std::unique_ptr<unsigned long long, cudaError_t (*)(void *)> guard(dCount, cudaFree);
    IBS_CUDA(cudaMemset(dCount, 0, sizeof *dCount), "count init");
    const int grid = grid_for(n, 256);
    if (t->geom.format == FMT_B8X32)
        k_count_present<FMT_B8X32><<<grid, 256>>>(t->view(), dCodes, n, dCount);
    else if (t->geom.format == FMT_MZ8)
        k_count_present<FMT_MZ8><<<grid, 256>>>(t->view(), dCodes, n, dCount);
    else if (t->geom.format == FMT_MZ6)
        k_count_present<FMT_MZ6><<<grid, 256>>>(t->view(), dCodes, n, dCount);
    else
        k_count_present<FMT_B6X40><<<grid, 256>>>(t->view(), dCodes, n, dCount);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "count launch");
    unsigned long long c = 0;
    IBS_CUDA(cudaMemcpy(&c, dCount, sizeof c, cudaMemcpyDeviceToHost), "count read");
    *count = c;
    return IBS_OK;
}

extern "C" ibs_status ibs_count_present(ibs_table *t, const uint64_t *codes, uint64_t n, int codes_on_device,
                                        uint64_t *count)
{
    clear_error();
    if (!t || !count || (n && !codes)) {
        set_error("ibs_count_present: bad argument");
        return IBS_ERR_ARG;
    }
    if (t->geom.format == FMT_WIDE) {
        set_error("ibs_count_present: takes the 64-bit codes of k <= 32 tables (a wide-key table counts "
                  "through ibs_count_present_kmc)");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(t->device);
    if (codes_on_device || !n)
        return count_present_device(t, codes, n, count);
    uint64_t *d = nullptr;
    IBS_CUDA(cudaMalloc(&d, n * 8), "codes alloc");
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> guard2(d, cudaFree);
    IBS_CUDA(cudaMemcpy(d, codes, n * 8, cudaMemcpyHostToDevice), "codes upload");
    return count_present_device(t, d, n, count);
}

extern "C" ibs_status ibs_count_present_kmc(ibs_table *t, const char *kmc_prefix, uint64_t *count)
{
    clear_error();
    if (!t || !kmc_prefix || !count) {
        set_error("ibs_count_present_kmc: bad argument");
        return IBS_ERR_ARG;
    }
    DeviceGuard guard(t->device);
    uint64_t *d = nullptr, n = 0;
    uint32_t k = 0;
    ibs_status s = decode_kmc_any(kmc_prefix, t->device, &d, &n, &k);
    if (s != IBS_OK)
        return s;
    std::unique_ptr<uint64_t, cudaError_t (*)(void *)> guard2(d, cudaFree);
    if (k != t->geom.k) {
        set_error("K-mer lengths do not match");
        return IBS_ERR_ARG;
    }
    if (t->geom.format == FMT_WIDE)
        return count_present_wide(t, reinterpret_cast<const ulonglong2 *>(d), n, count);
    return count_present_device(t, d, n, count);
}

extern "C" uint64_t ibs_table_bytes_for(uint64_t n_keys, uint32_t k, const ibs_table_opts *opts)
{
    if (k == 0 || k > kMaxWideK)
        return 0;
    if (k > 32) {
        // level 0 at the load, plus about 1% for the later levels
        const double lam = (opts && opts->keys_per_bucket > 0) ? opts->keys_per_bucket : 4.0;
        const uint64_t lines = (uint64_t)((double)n_keys / lam) + 1;
        return (lines + lines / 100 + 1) * wide::kSlots * 16;
    }
    return choose_geometry(n_keys, k, opts).nBuckets * 32;
}

extern "C" ibs_status ibs_device_memory(int device, uint64_t *free_bytes, uint64_t *total_bytes)
{
    clear_error();
    ibs_status s = check_device_ordinal(device);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(device);
    size_t f = 0, t = 0;
    IBS_CUDA(cudaMemGetInfo(&f, &t), "cudaMemGetInfo");
    if (free_bytes)
        *free_bytes = f;
    if (total_bytes)
        *total_bytes = t;
    return IBS_OK;
}

extern "C" void ibs_close(ibs_table *t)
{
    if (!t)
        return;
    {
        DeviceGuard guard(t->device);
        cudaFree(t->buckets);
        cudaFree(t->stash);
        free_wide(t);
    }
    delete t;
}
