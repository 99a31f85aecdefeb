// Internal declarations of libibs: error plumbing, the handle structs behind
// the C-ABI, and the device-side table lookup shared by every scan kernel.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/ibs.h"
#include "ibs_core.cuh"
#include "mz_core.cuh"
#include "wide_core.cuh"

namespace ibs {

// ---- errors ---------------------------------------------------------------
void set_error(const std::string &msg);
void clear_error();
std::atomic<uint64_t> &launch_counter();

// "CUDA error in <what>: <text>", the reference's message shape
// (src/gpu/EncodeProbe.cu:15-20).
ibs_status cuda_fail(cudaError_t e, const char *what);

#define IBS_CUDA(call, what)                                  \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess)                                \
            return ::ibs::cuda_fail(e_, what);                \
    } while (0)

// Device count check shared by the entry points.
ibs_status check_device_ordinal(int dev);
// Rows carry 32-bit window coordinates (ibs_window.start / end, the
// reference's int Window::start / end, src/Window.hpp:11-12), so a contig
// longer than INT32_MAX bases would print wrapped, negative coordinates:
// IBS_ERR_ARG with a message naming the contig instead.
ibs_status check_contig_lengths(const uint64_t *lens, uint32_t n, const char *what);
constexpr uint64_t kMaxContigLen = 2147483647ull;
// Decodes a KMC 3 database into canonical codes in device memory (caller
// frees). decode_kmc takes k <= 32 (one word per code); decode_kmc_any also
// takes 33 <= k <= 64, whose codes are two words each ({lo, hi}).
ibs_status decode_kmc(const char *prefix, int dev, uint64_t **dCodes, uint64_t *n, uint32_t *k);
ibs_status decode_kmc_any(const char *prefix, int dev, uint64_t **dCodes, uint64_t *n, uint32_t *k);
// Wide-key tables (ibs_wide.cu): the build from device codes ({lo, hi} per
// key; the device must be current), membership counts, and the release of
// the levels.
ibs_status build_wide(ibs_table *t, const ulonglong2 *dCodes, uint64_t n, uint32_t k, const ibs_table_opts *o);
ibs_status count_present_wide(ibs_table *t, const ulonglong2 *dCodes, uint64_t n, uint64_t *count);
void free_wide(ibs_table *t);
constexpr uint32_t kMaxWideK = 64;
// Packed base offset of each contig (roundup64 of the lengths before it) and
// the seq / mask word counts with their tail padding.
void packed_offsets(const uint64_t *lens, uint32_t n, std::vector<uint64_t> &off, uint64_t &seqWords,
                    uint64_t &maskWords);
// A reference around device arrays already in the packed layout; it takes
// ownership of dSeq / dMask (freed by ibs_reference_free, also on failure).
ibs_status reference_adopt(const std::vector<uint64_t> &lens, int device, uint64_t *dSeq, uint64_t *dMask,
                           ibs_reference **out);

#define IBS_LAUNCHED() (::ibs::launch_counter().fetch_add(1, std::memory_order_relaxed))

// RAII guard that makes `dev` current and restores the previous device.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess)
            prev = -1;
        ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard()
    {
        if (prev >= 0)
            cudaSetDevice(prev);
    }
};

// ---- tuning -----------------------------------------------------------------
const ibs_tuning &tuning();

// ---- device table view ----------------------------------------------------
struct TableView {
    TableGeom g;
    const uint4 *buckets; // 2 x uint4 per bucket
    const uint64_t *stash;
};

#if defined(__CUDACC__)
__device__ __forceinline__ bool stash_lookup(const TableView &t, uint64_t code)
{
    if (t.g.stashBuckets == 0)
        return false;
    uint64_t b = stash_home(code, t.g.stashBuckets);
    for (uint64_t i = 0; i < t.g.stashBuckets; ++i) {
        const ulonglong2 *p = reinterpret_cast<const ulonglong2 *>(t.stash + 4 * b);
        const ulonglong2 a = __ldg(p), c = __ldg(p + 1);
        if (a.x == code || a.y == code || c.x == code || c.y == code)
            return true;
        if (a.x == STASH_EMPTY || a.y == STASH_EMPTY || c.x == STASH_EMPTY || c.y == STASH_EMPTY)
            return false;
        b = (b + 1) & (t.g.stashBuckets - 1);
    }
    return false;
}

// One bucket compare, given the bucket's two 16-byte halves. Returns 1 on a
// hit, 0 on a sure miss, 2 when the bucket overflowed into the stash.
template <uint32_t FMT>
__device__ __forceinline__ uint32_t bucket_match(const uint4 &v0, const uint4 &v1, uint64_t fp)
{
    if (FMT == FMT_B8X32) {
        const uint32_t f = (uint32_t)fp;
        const bool hit = (v0.x == f) | (v0.y == f) | (v0.z == f) | (v0.w == f) | (v1.x == f) |
                         (v1.y == f) | (v1.z == f) | (v1.w == f);
        return hit ? 1u : (v1.w == B8_OVERFLOW ? 2u : 0u);
    } else {
        const uint32_t qhi = (uint32_t)(fp >> 8), qlo = (uint32_t)(fp & 0xff);
        const uint32_t cnt = (v1.w >> 16) & 0xff;
        bool hit = false;
        hit |= (0 < cnt) & (v0.x == qhi) & ((v1.z & 0xff) == qlo);
        hit |= (1 < cnt) & (v0.y == qhi) & (((v1.z >> 8) & 0xff) == qlo);
        hit |= (2 < cnt) & (v0.z == qhi) & (((v1.z >> 16) & 0xff) == qlo);
        hit |= (3 < cnt) & (v0.w == qhi) & ((v1.z >> 24) == qlo);
        hit |= (4 < cnt) & (v1.x == qhi) & ((v1.w & 0xff) == qlo);
        hit |= (5 < cnt) & (v1.y == qhi) & (((v1.w >> 8) & 0xff) == qlo);
        return hit ? 1u : ((v1.w >> 24) & 1u ? 2u : 0u);
    }
}

// An MZ8 sector compare: 1 on a hit, 0 on a sure miss, 2 when the sector's
// extra keys are in its partner sector, 3 when also in the stash.
__device__ __forceinline__ uint32_t mz8_match(const uint4 &v0, const uint4 &v1, uint32_t slot)
{
    const bool hit = (v0.x == slot) | (v0.y == slot) | (v0.z == slot) | (v0.w == slot) | (v1.x == slot) |
                     (v1.y == slot) | (v1.z == slot) | (v1.w == slot);
    return hit ? 1u : (v1.w == B8_OVERFLOW ? 2u : (v1.w == B8_OVERFLOW_STASH ? 3u : 0u));
}

// The rest of an MZ8 probe whose sector r reported m >= 2: the partner
// sector r ^ 1 of the same line, then (m == 3) the stash.
__device__ __forceinline__ bool mz8_overflow_lookup(const TableView &t, uint64_t r, uint32_t slot, uint32_t m,
                                                    uint64_t code)
{
    const uint4 w0 = __ldg(t.buckets + 2 * (r ^ 1)), w1 = __ldg(t.buckets + 2 * (r ^ 1) + 1);
    if ((w0.x == slot) | (w0.y == slot) | (w0.z == slot) | (w0.w == slot) | (w1.x == slot) | (w1.y == slot) |
        (w1.z == slot) | (w1.w == slot))
        return true;
    return m == 3u && stash_lookup(t, code);
}

template <uint32_t FMT>
__device__ __forceinline__ bool table_lookup(const TableView &t, uint64_t code)
{
    if (FMT == FMT_MZ8) {
        uint64_t r, slot;
        mz::locate(code, t.g, r, slot);
        const uint4 v0 = __ldg(t.buckets + 2 * r), v1 = __ldg(t.buckets + 2 * r + 1);
        const uint32_t m = mz8_match(v0, v1, (uint32_t)slot);
        return m == 1u || (m >= 2u && mz8_overflow_lookup(t, r, (uint32_t)slot, m, code));
    }
    if (FMT == FMT_MZ6) {
        uint64_t r, slot;
        mz::locate(code, t.g, r, slot);
        const uint4 v0 = __ldg(t.buckets + 2 * r), v1 = __ldg(t.buckets + 2 * r + 1);
        const uint32_t m = bucket_match<FMT_B6X40>(v0, v1, slot);
        return m == 1u || (m == 2u && stash_lookup(t, code));
    }
    const uint64_t h = perm_hash(code, t.g.bits);
    const uint64_t r = bucket_of(h, t.g);
    const uint4 v0 = __ldg(t.buckets + 2 * r), v1 = __ldg(t.buckets + 2 * r + 1);
    const uint32_t m = bucket_match<FMT>(v0, v1, fp_of(h, t.g));
    return m == 1u || (m == 2u && stash_lookup(t, code));
}
#endif

} // namespace ibs

// ---- handles ----------------------------------------------------------------
struct ibs_table {
    int device = 0;
    ibs::TableGeom geom{};
    uint4 *buckets = nullptr;
    uint64_t *stash = nullptr;
    uint64_t nKeys = 0, stashKeys = 0;
    double buildSeconds = 0;
    uint64_t deviceBytes = 0;
    ibs::wide::View wide{}; // the levels of a wide-key table (geom.format == FMT_WIDE)
    ibs::TableView view() const { return ibs::TableView{geom, buckets, stash}; }
};

namespace ibs {
// Per-window descriptor on the device.
struct WinDesc {
    uint64_t base; // packed base offset of the window's first base
    uint32_t nPos; // k-mer positions
    int32_t start, end;
    uint32_t pad;
};

// Windows, spans and scratch of one (reference, W, k, span length) plan.
struct ScanPlan {
    uint32_t W = 0, k = 0, spanLen = 0;
    uint64_t nWin = 0, nSpans = 0;
    std::vector<WinDesc> win;     // host copy
    std::vector<uint32_t> span0;  // host copy, nWin + 1
    WinDesc *dWin = nullptr;
    uint32_t *dSpan0 = nullptr;
    SegStats *dSpans = nullptr;   // scratch: one summary per span
    void release();
};

// Build the plan's host arrays for contigs `lens` starting at packed
// offsets `baseOff`.
void plan_windows(ScanPlan &p, const std::vector<uint64_t> &lens,
                  const std::vector<uint64_t> &baseOff, uint32_t W, uint32_t k, uint32_t spanLen);

// Launch the span kernel over spans [s0, s1) and, when fin, the window
// finalizer over every window of the plan.
ibs_status launch_scan(const ibs_table *t, const uint64_t *dSeq, const uint64_t *dMask,
                       const ScanPlan &p, uint64_t s0, uint64_t s1, cudaStream_t st);
ibs_status launch_finalize(const ScanPlan &p, uint32_t k, ibs_window *dRows, cudaStream_t st);
ibs_status launch_panel(ibs_table *const *tables, uint32_t nTables, const uint64_t *dSeq,
                        const uint64_t *dMask, const ScanPlan &p, ibs_window *dRows,
                        SegStats *dSpans, cudaStream_t st);
} // namespace ibs

struct ibs_reference {
    int device = 0;
    std::vector<uint64_t> lens, baseOff;
    std::vector<std::string> ids;       // contig ids when parsed from FASTA by the library
    uint64_t seqWords = 0, maskWords = 0;
    uint64_t *dSeq = nullptr, *dMask = nullptr;
    ibs::ScanPlan plan;                 // cached for the last (W, k)
    ibs_window *dRows = nullptr;        // cached row buffer for ibs_scan
    uint64_t dRowsCap = 0;
    ibs::SegStats *dPanelSpans = nullptr; // panel scratch
    uint64_t dPanelSpansCap = 0;
    cudaStream_t stream = nullptr;
};
