// Wide-key tables (33 <= k <= 64): the level-by-level build, membership
// probes and counts. Layout and lookup rule in wide_core.cuh.
//
// The reference has no device table for these k: its string path looks each
// canonical k-mer string up in the KMC database on the host
// (getStatsFromSequenceLegacy, src/KmerDatabase.hpp:675-708; CKmerAPI::
// from_string + CKMCFile::IsKmer). The build here is a counting placement:
// per level, every key counts its line, lines with more than 8 keys send the
// surplus to the next level's input, and every key then claims a slot of its
// line in arrival order (the first 8 of a line stay; which 8 does not
// matter to membership).
#include "ibs_internal.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <vector>

namespace ibs {
namespace {

using wide::kEmpty;
using wide::kSlots;

__device__ __forceinline__ bool is_empty_key(const ulonglong2 &v) { return v.x == kEmpty && v.y == kEmpty; }

__global__ void k_wcount(const ulonglong2 *__restrict__ keys, uint64_t n, uint32_t level, uint64_t lines,
                         uint32_t *__restrict__ cnt)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 v = keys[i];
        if (!is_empty_key(v))
            atomicAdd(cnt + wide::line_of(v.x, v.y, level, lines), 1u);
    }
}

// Keys beyond kSlots per line (the next level's input), summed; resets the
// counters for the placement pass.
__global__ void k_wover(uint32_t *__restrict__ cnt, uint64_t lines, unsigned long long *__restrict__ over)
{
    unsigned long long local = 0;
    for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < lines;
         r += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t c = cnt[r];
        if (c > kSlots)
            local += c - kSlots;
        cnt[r] = 0;
    }
    for (int o = 16; o; o >>= 1)
        local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local)
        atomicAdd(over, local);
}

__global__ void k_wplace(const ulonglong2 *__restrict__ keys, uint64_t n, uint32_t level, uint64_t lines,
                         uint32_t *__restrict__ cnt, ulonglong2 *__restrict__ slots, ulonglong2 *__restrict__ next,
                         unsigned long long *__restrict__ nextN, uint64_t nextCap, int *__restrict__ err)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 v = keys[i];
        if (is_empty_key(v))
            continue;
        const uint64_t r = wide::line_of(v.x, v.y, level, lines);
        const uint32_t s = atomicAdd(cnt + r, 1u);
        if (s < kSlots) {
            slots[r * kSlots + s] = v;
        } else {
            const unsigned long long j = atomicAdd(nextN, 1ull);
            if (j < nextCap)
                next[j] = v;
            else
                atomicExch(err, 1);
        }
    }
}

__global__ void k_wprobe(wide::View t, const ulonglong2 *__restrict__ keys, uint64_t n, uint8_t *__restrict__ hits)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 v = keys[i];
        hits[i] = wide::lookup(t, v.x, v.y) ? 1 : 0;
    }
}

__global__ void k_wcount_present(wide::View t, const ulonglong2 *__restrict__ keys, uint64_t n,
                                 unsigned long long *__restrict__ count)
{
    unsigned long long local = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const ulonglong2 v = keys[i];
        local += wide::lookup(t, v.x, v.y) ? 1 : 0;
    }
    for (int o = 16; o; o >>= 1)
        local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0 && local)
        atomicAdd(count, local);
}

int grid_of(uint64_t n, int threads)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + threads - 1) / threads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 16));
}

template <typename T> struct DevPtr {
    T *p = nullptr;
    DevPtr() = default;
    DevPtr(const DevPtr &) = delete;
    DevPtr &operator=(const DevPtr &) = delete;
    ~DevPtr() { cudaFree(p); }
    cudaError_t alloc(uint64_t n) { return cudaMalloc(&p, std::max<uint64_t>(n, 1) * sizeof(T)); }
};

bool key_less(const ibs_code128 &a, const ibs_code128 &b) { return a.hi != b.hi ? a.hi < b.hi : a.lo < b.lo; }
bool key_eq(const ibs_code128 &a, const ibs_code128 &b) { return a.hi == b.hi && a.lo == b.lo; }

ibs_status check_wide_k(uint32_t k, const char *what)
{
    if (k <= 32 || k > kMaxWideK) {
        set_error(std::string(what) + ": wide-key tables need 33 <= k <= 64 (k=" + std::to_string(k) + ")");
        return k > kMaxWideK ? IBS_ERR_UNSUPPORTED : IBS_ERR_ARG;
    }
    return IBS_OK;
}

} // namespace

void free_wide(ibs_table *t)
{
    for (uint32_t L = 0; L < wide::kMaxLevels; ++L) {
        cudaFree(const_cast<ulonglong2 *>(t->wide.slots[L]));
        t->wide.slots[L] = nullptr;
    }
    t->wide.nLevels = 0;
}

ibs_status build_wide(ibs_table *t, const ulonglong2 *dCodes, uint64_t n, uint32_t k, const ibs_table_opts *o)
{
    ibs_status s = check_wide_k(k, "wide-key table");
    if (s != IBS_OK)
        return s;
    if (o && o->force_format && o->force_format != FMT_WIDE) {
        set_error("k=" + std::to_string(k) + " > 32 takes only the wide-key table layout (format 8)");
        return IBS_ERR_UNSUPPORTED;
    }
    const double lam = (o && o->keys_per_bucket > 0) ? o->keys_per_bucket : 4.0; // keys per 128-byte line
    t->geom = TableGeom{};
    t->geom.k = k;
    t->geom.bits = 2 * k;
    t->geom.format = FMT_WIDE;
    t->nKeys = n;
    t->wide = wide::View{};
    t->wide.k = k;
    const uint64_t lines0 = std::max<uint64_t>(1, (uint64_t)((double)n / lam) + 1);
    DevPtr<uint32_t> cnt; // per line of the level; cntCap lines
    uint64_t cntCap = lines0;
    DevPtr<unsigned long long> dOver; // [0] surplus keys of the level, [1] next-level fill
    DevPtr<int> dErr;
    IBS_CUDA(cnt.alloc(cntCap), "wide table scratch");
    IBS_CUDA(dOver.alloc(2), "wide table scratch");
    IBS_CUDA(dErr.alloc(1), "wide table scratch");
    IBS_CUDA(cudaMemset(dErr.p, 0, sizeof(int)), "wide table scratch");
    // cur: this level's input (the caller's codes, then the surplus of the
    // previous level, held by owned)
    const ulonglong2 *cur = dCodes;
    uint64_t nCur = n;
    std::unique_ptr<DevPtr<ulonglong2>> owned;
    uint64_t bytes = 0, stashKeys = 0;
    for (uint32_t L = 0;; ++L) {
        if (L == wide::kMaxLevels) {
            set_error("wide-key table: keys left after " + std::to_string(wide::kMaxLevels) +
                      " levels (duplicate keys in the input?)");
            return IBS_ERR_CAPACITY;
        }
        const uint64_t lines = L == 0 ? lines0 : std::max<uint64_t>(1, (nCur + 1) / 2);
        if (lines > cntCap) {
            cudaFree(cnt.p);
            cnt.p = nullptr;
            cntCap = lines;
            IBS_CUDA(cnt.alloc(cntCap), "wide table scratch");
        }
        ulonglong2 *slots = nullptr;
        IBS_CUDA(cudaMalloc(&slots, lines * kSlots * sizeof(ulonglong2)), "wide table alloc");
        t->wide.slots[L] = slots;
        t->wide.lines[L] = lines;
        t->wide.nLevels = L + 1;
        bytes += lines * kSlots * sizeof(ulonglong2);
        IBS_CUDA(cudaMemset(slots, 0xff, lines * kSlots * sizeof(ulonglong2)), "wide table init");
        IBS_CUDA(cudaMemset(cnt.p, 0, lines * sizeof(uint32_t)), "wide table counts");
        IBS_CUDA(cudaMemset(dOver.p, 0, 2 * sizeof(unsigned long long)), "wide table counts");
        if (nCur) {
            k_wcount<<<grid_of(nCur, 256), 256>>>(cur, nCur, L, lines, cnt.p);
            IBS_LAUNCHED();
        }
        k_wover<<<grid_of(lines, 256), 256>>>(cnt.p, lines, dOver.p);
        IBS_LAUNCHED();
        unsigned long long over = 0;
        IBS_CUDA(cudaMemcpy(&over, dOver.p, sizeof over, cudaMemcpyDeviceToHost), "wide table count");
        std::unique_ptr<DevPtr<ulonglong2>> next(new DevPtr<ulonglong2>);
        if (over)
            IBS_CUDA(next->alloc(over), "wide table level input");
        if (nCur) {
            k_wplace<<<grid_of(nCur, 256), 256>>>(cur, nCur, L, lines, cnt.p, slots, next->p, dOver.p + 1, over,
                                                  dErr.p);
            IBS_LAUNCHED();
        }
        int herr = 0;
        IBS_CUDA(cudaMemcpy(&herr, dErr.p, sizeof herr, cudaMemcpyDeviceToHost), "wide table place");
        if (herr) {
            set_error("wide-key table: level input overran its count");
            return IBS_ERR_CAPACITY;
        }
        if (L == 0)
            stashKeys = over; // every key past level 0 stays in a later level
        owned = std::move(next);
        cur = owned->p;
        nCur = over;
        if (!over)
            break;
    }
    t->geom.nBuckets = 0;
    for (uint32_t L = 0; L < t->wide.nLevels; ++L)
        t->geom.nBuckets += t->wide.lines[L] * 4; // in 32-byte units, as the other formats report
    t->stashKeys = stashKeys;                     // keys held by levels past the first
    t->deviceBytes = bytes;
    return IBS_OK;
}

ibs_status count_present_wide(ibs_table *t, const ulonglong2 *dCodes, uint64_t n, uint64_t *count)
{
    *count = 0;
    if (!n)
        return IBS_OK;
    DevPtr<unsigned long long> dCount;
    IBS_CUDA(dCount.alloc(1), "count alloc");
    IBS_CUDA(cudaMemset(dCount.p, 0, sizeof(unsigned long long)), "count init");
    k_wcount_present<<<grid_of(n, 256), 256>>>(t->wide, dCodes, n, dCount.p);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "count launch");
    unsigned long long c = 0;
    IBS_CUDA(cudaMemcpy(&c, dCount.p, sizeof c, cudaMemcpyDeviceToHost), "count read");
    *count = c;
    return IBS_OK;
}

} // namespace ibs

using namespace ibs;

extern "C" ibs_status ibs_table_from_codes128(const ibs_code128 *codes, uint64_t n, uint32_t k, int codes_on_device,
                                              const ibs_table_opts *opts, ibs_table **out)
{
    clear_error();
    if (!out || (!codes && n)) {
        set_error("ibs_table_from_codes128: bad argument");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    ibs_status s = check_wide_k(k, "ibs_table_from_codes128");
    if (s != IBS_OK)
        return s;
    const int dev = opts ? opts->device : 0;
    s = check_device_ordinal(dev);
    if (s != IBS_OK)
        return s;
    DeviceGuard guard(dev);
    const auto t0 = std::chrono::steady_clock::now();
    // duplicates removed on the host (a key repeated more than 8 times per
    // level would never leave the level chain)
    std::vector<ibs_code128> keys(n);
    if (n) {
        if (codes_on_device)
            IBS_CUDA(cudaMemcpy(keys.data(), codes, n * sizeof(ibs_code128), cudaMemcpyDeviceToHost), "codes download");
        else
            memcpy(keys.data(), codes, n * sizeof(ibs_code128));
    }
    std::sort(keys.begin(), keys.end(), key_less);
    keys.erase(std::unique(keys.begin(), keys.end(), key_eq), keys.end());
    const uint64_t m = keys.size();
    DevPtr<ulonglong2> d;
    IBS_CUDA(d.alloc(m), "codes alloc");
    if (m)
        IBS_CUDA(cudaMemcpy(d.p, keys.data(), m * sizeof(ibs_code128), cudaMemcpyHostToDevice), "codes upload");
    std::unique_ptr<ibs_table> t(new ibs_table);
    t->device = dev;
    s = build_wide(t.get(), d.p, m, k, opts);
    if (s != IBS_OK) {
        ibs_close(t.release());
        return s;
    }
    t->buildSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = t.release();
    return IBS_OK;
}

extern "C" ibs_status ibs_probe128(ibs_table *t, const ibs_code128 *codes, uint64_t n, uint8_t *hits)
{
    clear_error();
    if (!t || (n && (!codes || !hits))) {
        set_error("ibs_probe128: bad argument");
        return IBS_ERR_ARG;
    }
    if (t->geom.format != FMT_WIDE) {
        set_error("ibs_probe128: the table is not a wide-key table (k <= 32 tables take ibs_probe)");
        return IBS_ERR_ARG;
    }
    if (!n)
        return IBS_OK;
    DeviceGuard guard(t->device);
    DevPtr<ulonglong2> dCodes;
    DevPtr<uint8_t> dHits;
    IBS_CUDA(dCodes.alloc(n), "probe alloc");
    IBS_CUDA(dHits.alloc(n), "probe alloc");
    IBS_CUDA(cudaMemcpy(dCodes.p, codes, n * sizeof(ibs_code128), cudaMemcpyHostToDevice), "probe upload");
    k_wprobe<<<grid_of(n, 256), 256>>>(t->wide, dCodes.p, n, dHits.p);
    IBS_LAUNCHED();
    IBS_CUDA(cudaGetLastError(), "probe launch");
    IBS_CUDA(cudaMemcpy(hits, dHits.p, n, cudaMemcpyDeviceToHost), "probe");
    return IBS_OK;
}
