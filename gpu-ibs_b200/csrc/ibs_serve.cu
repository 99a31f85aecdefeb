// The serving loop: continuous batching of window-scan requests.
//
// A request names a sample and a range of windows of one contig. Samples
// live in device tables, here called groups: a single-sample table (the
// minimizer-line formats MZ8 / MZ6 or the hash formats B8x32 / B6x40; the
// server builds them in its table_format option's layout) or a joint panel
// table (P5x48, one sample-mask per key, up to 16 samples). Windows are numbered across contigs, so a request
// is an interval of that numbering.
//
// A background thread runs iterations. Each one admits new requests, makes
// the groups they need resident (least-recently-used eviction under a byte
// budget, reload from a pinned host image on a side stream) and then, for
// every resident group with pending windows, takes the next run of pending
// windows from that group's sweep cursor. Each such window is scanned ONCE
// for all the pending requests that contain it: in a joint table one bucket
// load per position answers every requesting sample, and two requests of one
// sample share the scan. The span kernels write one statistics summary per
// (span, requesting sample); the finalizer folds each (request, window)'s
// summaries into that request's row. Two iterations are in flight at a time
// and a request submitted meanwhile joins the next one. A request's rows are
// the same windows' rows of a full scan of its sample, whatever it was
// batched with.
//
// With one_request_per_launch an iteration runs the windows of one request
// only, against its own table: the plain path, one launch per request.
//
// No device code waits on the host: each launch is a finite kernel over a
// finite work list.
#include "mz_scan.cuh"
#include "panel_core.cuh"
#include "scan_device.cuh"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace ibs {
namespace serve {

constexpr uint32_t kSpanLen = 4096;
constexpr int kNB = 4;
constexpr uint64_t kSumCap = 1ull << 20;   // span summaries per launch (32 B each): 32 MiB
constexpr uint64_t kPosCap = 512ull << 20; // reference positions scanned per launch
constexpr uint64_t kFinCap = 1ull << 20;   // (request, window) rows finalized per launch
constexpr uint64_t kRowPool = 4ull << 20;  // rows of admitted requests (24 B each): 96 MiB
constexpr uint32_t kMaxGroups = 4096;
constexpr int kDepth = 4;                  // iterations (batches) in flight
constexpr int kServeNB = 2;                // blocks in flight per lane of the single-table kernel (64
                                           // registers, four CTAs of 256 per SM) and of the persistent
                                           // kernel (80 registers without spills, three CTAs per SM)

struct WorkItem {
    uint64_t base;   // packed base offset of the window's first base
    uint32_t p0, p1; // positions of the window
    uint32_t view;   // index into this launch's views of its kind
    uint32_t mask;   // requesting samples (bits of a joint table; 1 for a single table)
    uint64_t out;    // first summary slot; sample of rank i writes out + i
};

struct FinItem {
    uint64_t sum;    // summary of the window's first span for this request's sample
    uint32_t nSpans, stride;
    int32_t start, end;
    uint64_t row;    // row slot
};

// One work item over a single-sample table, by one warp: the summary of
// positions [p0, p1) of its window goes to sums[it.out]. Minimizer-line
// tables (MZ8, MZ6) take the window scan's minimizer path
// (dev::mz_span_stats), the hash-bucket tables one bucket load per
// position. K > 0 is the server's k fixed at compile time (0: read from the
// table).
template <int NB, uint32_t K>
__device__ __forceinline__ void serve_single_item(const WorkItem &it, const TableView &t,
                                                  const uint64_t *__restrict__ seq,
                                                  const uint64_t *__restrict__ mask, SegStats *__restrict__ sums,
                                                  uint32_t lane)
{
    if (is_mz(t.g.format)) {
        // the span's m-mer reads stop at its last position's last m-mer,
        // inside the window's bases
        const uint32_t lastM = it.p1 - 1 + (mz::w_of(K ? K : t.g.k) - 1);
        const SegStats acc =
            t.g.format == FMT_MZ8
                ? dev::mz_span_stats<NB, K, FMT_B8X32>(t, seq, mask, it.base, it.p0, it.p1, lastM, lane)
                : dev::mz_span_stats<NB, K, FMT_B6X40>(t, seq, mask, it.base, it.p0, it.p1, lastM, lane);
        if (lane == 0)
            sums[it.out] = acc;
        return;
    }
    const uint32_t k = t.g.k;
    const uint64_t kmask = key_mask(2 * k);
    const uint64_t kbits = (1ull << k) - 1;
    const bool b8 = t.g.format == FMT_B8X32;
    dev::LaneFold fold;
    for (uint32_t p = it.p0; p < it.p1; p += 32 * NB) {
        uint4 v0[NB], v1[NB];
        uint64_t code[NB], fp[NB];
        bool valid[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const uint32_t q = p + 32 * b + lane;
            const bool in = q < it.p1;
            const uint64_t G = it.base + (in ? q : it.p0);
            bool acgt;
            code[b] = dev::canonical_at(seq, mask, G, k, kmask, kbits, acgt);
            valid[b] = in && acgt;
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
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            bool hit = false;
            if (valid[b]) {
                const uint32_t m = b8 ? bucket_match<FMT_B8X32>(v0[b], v1[b], fp[b])
                                      : bucket_match<FMT_B6X40>(v0[b], v1[b], fp[b]);
                hit = m == 1u || (m == 2u && stash_lookup(t, code[b]));
            }
            const uint32_t V = __ballot_sync(dev::FULL_MASK, valid[b]);
            const uint32_t H = __ballot_sync(dev::FULL_MASK, hit);
            fold.push(V, H, lane, (int)k);
        }
    }
    const SegStats acc = fold.finish((int)k);
    if (lane == 0)
        sums[it.out] = acc;
}

// A run of up to 32 blocks of one sample, lane i holding block i's valid
// (v) and hit (h) masks (empty past the run): the run's statistics, appended
// to acc in lane 0 (the plain scan's lane-parallel fold, dev::LaneFold,
// without its own accumulator).
__device__ __forceinline__ void fold_run_into(SegStats &acc, uint32_t v, uint32_t h, int k)
{
    Seg32 s = block_seg32(v, h, k);
#pragma unroll
    for (uint32_t off = 1; off < 32; off <<= 1) {
        Seg32 o;
        o.total = __shfl_down_sync(dev::FULL_MASK, s.total, off);
        o.obs = __shfl_down_sync(dev::FULL_MASK, s.obs, off);
        o.lead = __shfl_down_sync(dev::FULL_MASK, s.lead, off);
        o.trail = __shfl_down_sync(dev::FULL_MASK, s.trail, off);
        o.gaps = __shfl_down_sync(dev::FULL_MASK, s.gaps, off);
        o.dist = __shfl_down_sync(dev::FULL_MASK, s.dist, off);
        s = seg32_combine(s, o, k);
    }
    acc = seg_combine(acc, seg_of(s), k);
}

// One work item over a joint table: one bucket load per position; lane j
// keeps the statistics of sample j when j is in the item's mask, and the
// requesting samples' summaries go to sums[it.out + rank]. An item that
// requests one sample (a lone request's windows) folds it lane-parallel
// instead: lane i keeps block i of every 32 and the run is summarised at
// once, where the per-sample serial block summaries would leave 31 lanes
// idle. K > 0 is the server's k, which every table of the server has (the
// server refuses a table of another k): the minimizer window and masks are
// then compile-time, and the minimizer-line layout is pruned where k rules
// it out.
template <int NB, uint32_t K = 0>
__device__ __forceinline__ void serve_joint_item(const WorkItem &it, const panel::View &t,
                                                 const uint64_t *__restrict__ seq,
                                                 const uint64_t *__restrict__ mask, SegStats *__restrict__ sums,
                                                 uint32_t lane)
{
    const uint32_t k = K ? K : t.g.k;
    const uint64_t kmask = key_mask(2 * k);
    const uint64_t kbits = (1ull << k) - 1;
    const uint32_t want = it.mask & 0xffffu;
    const bool one = (want & (want - 1u)) == 0u; // warp-uniform
    const uint32_t j0 = __ffs(want) - 1;
    // minimizer-line joint tables (PM) locate a k-mer through its minimizer:
    // m-mers read one block ahead, up to the span's last position's last
    // m-mer (inside the window's bases); that layout exists only for
    // 16 <= k <= 27
    constexpr bool kPmPossible = K == 0 || (K >= 16 && K <= 27);
    const bool pm = kPmPossible && t.g.format == FMT_PANEL_MZ;
    const uint32_t w = pm ? mz::w_of(k) : 1, m = pm ? mz::m_of(k) : 0;
    const uint32_t lastM = it.p1 - 1 + (w - 1);
    dev::MzPos next;
    if (pm)
        next = dev::mz_pos(seq, mask, it.base + min(it.p0 + lane, lastM), k, m);
    SegStats acc = seg_empty();
    uint32_t fv = 0, fh = 0; // one sample: this lane's block of the current run
    for (uint32_t p = it.p0; p < it.p1; p += 32 * NB) {
        uint4 v0[NB], v1[NB];
        uint64_t code[NB], rr[NB];
        uint32_t fp[NB];
        bool valid[NB];
        if (pm) {
            dev::MzPos ps[NB + 1];
            ps[0] = next;
#pragma unroll
            for (int b = 1; b <= NB; ++b)
                ps[b] = dev::mz_pos(seq, mask, it.base + min(p + 32 * b + lane, lastM), k, m);
            next = ps[NB];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                valid[b] = p + 32 * b + lane < it.p1 && ps[b].acgt;
                uint64_t slot;
                dev::mz_locate_lane<true>(ps[b], ps[b + 1], lane, k, w, t.g.nBuckets, t.g.fpBits, rr[b], slot);
                fp[b] = (uint32_t)slot;
                code[b] = ps[b].code;
            }
        } else {
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                const uint32_t q = p + 32 * b + lane;
                const bool in = q < it.p1;
                const uint64_t G = it.base + (in ? q : it.p0);
                bool acgt;
                code[b] = dev::canonical_at(seq, mask, G, k, kmask, kbits, acgt);
                valid[b] = in && acgt;
                const uint64_t h = perm_hash(code[b], t.g.bits);
                rr[b] = bucket_of(h, t.g);
                fp[b] = (uint32_t)fp_of(h, t.g);
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (valid[b]) {
                v0[b] = __ldg(t.buckets + 2 * rr[b]);
                v1[b] = __ldg(t.buckets + 2 * rr[b] + 1);
            } else {
                v0[b] = make_uint4(0, 0, 0, 0);
                v1[b] = make_uint4(0, 0, 0, 0);
            }
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            uint32_t m = 0;
            if (valid[b]) {
                if (pm) {
                    m = panel::pm_mask(t, v0[b], v1[b], rr[b], fp[b], code[b]);
                } else {
                    m = panel::bucket_mask(v0[b], v1[b], fp[b]);
                    if (m & 0x80000000u)
                        m = panel::stash_mask(t, code[b]);
                }
            }
            const uint32_t V = __ballot_sync(dev::FULL_MASK, valid[b]);
            if (one) {
                const uint32_t H = __ballot_sync(dev::FULL_MASK, (m >> j0) & 1u);
                const uint32_t blk = (((p - it.p0) >> 5) + b) & 31u; // warp-uniform
                if (lane == blk) {
                    fv = V;
                    fh = H;
                }
                if (blk == 31u) {
                    fold_run_into(acc, fv, fh, (int)k);
                    fv = fh = 0;
                }
                continue;
            }
            uint32_t myH = 0;
            for (uint32_t rest = want; rest; rest &= rest - 1) { // warp-uniform
                const uint32_t j = __ffs(rest) - 1;
                const uint32_t Hj = __ballot_sync(dev::FULL_MASK, (m >> j) & 1u);
                if (lane == j)
                    myH = Hj;
            }
            if ((want >> lane) & 1u)
                acc = seg_combine(acc, panel::block_stats_serial(V, myH, (int)k), (int)k);
        }
    }
    if (one) {
        // the last, partial run (lanes past it hold empty blocks)
        if (__any_sync(dev::FULL_MASK, fv != 0))
            fold_run_into(acc, fv, fh, (int)k);
        if (lane == 0)
            sums[it.out] = acc;
        return;
    }
    if ((want >> lane) & 1u)
        sums[it.out + __popc(want & ((1u << lane) - 1u))] = acc;
}

// One (request, window) row from the window's span summaries.
__device__ __forceinline__ void serve_fin_item(const FinItem &f, const SegStats *__restrict__ sums, int k,
                                               ibs_window *__restrict__ rows)
{
    SegStats acc = seg_empty();
    for (uint32_t s = 0; s < f.nSpans; ++s)
        acc = seg_combine(acc, sums[f.sum + (uint64_t)s * f.stride], k);
    WindowRow row;
    row.start = f.start;
    row.end = f.end;
    seg_finish(acc, k, row);
    ibs_window o;
    o.start = row.start;
    o.end = row.end;
    o.total_kmers = row.total_kmers;
    o.observed_kmers = row.observed_kmers;
    o.variations = row.variations;
    o.kmer_distance = row.kmer_distance;
    rows[f.row] = o;
}

// ---- one launch per iteration (one_request_per_launch: the plain path) ----
template <int NB, uint32_t K>
__global__ void __launch_bounds__(256, 4) k_serve_single(const TableView *__restrict__ views,
                                                         const WorkItem *__restrict__ items, uint32_t nItems,
                                                         const uint64_t *__restrict__ seq,
                                                         const uint64_t *__restrict__ mask,
                                                         SegStats *__restrict__ sums)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < nItems; i += nWarps) {
        const WorkItem it = items[i];
        serve_single_item<NB, K>(it, views[it.view], seq, mask, sums, lane);
    }
}

template <int NB, uint32_t K>
__global__ void __launch_bounds__(256) k_serve_joint(const panel::View *__restrict__ views,
                                                     const WorkItem *__restrict__ items, uint32_t nItems,
                                                     const uint64_t *__restrict__ seq,
                                                     const uint64_t *__restrict__ mask,
                                                     SegStats *__restrict__ sums)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nWarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < nItems; i += nWarps) {
        const WorkItem it = items[i];
        serve_joint_item<NB, K>(it, views[it.view], seq, mask, sums, lane);
    }
}

__global__ void k_serve_finalize(const FinItem *__restrict__ fin, uint32_t n, const SegStats *__restrict__ sums,
                                 int k, ibs_window *__restrict__ rows)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        serve_fin_item(fin[i], sums, k, rows);
}

// ---- the persistent launch (batched serving) --------------------------------
// One kernel stays resident while requests keep arriving. The host publishes
// batches (the work of one loop iteration: span items over single and joint
// tables, then the rows to fold) into a ring of kRing descriptors in pinned
// host memory and raises `published`, a count of tickets. Warps claim
// tickets from a device counter in order: the scan tickets of a batch come
// first, one span item each, then its fold tickets, kFinPerTicket rows each.
// A fold ticket waits until the batch's scan items are done; the warp that
// completes a batch's last fold ticket stamps it done in pinned host memory,
// where the host loop sees it. Rows are written straight into the pinned
// row pool.
//
// Every wait is bounded. A warp whose ticket is not published within the
// idle limit stops the kernel (the host launches it again when work comes);
// a fold ticket whose batch's scans do not finish within the wait limit
// stops it with a timeout status. Batches that were published but not done
// when the kernel stopped are published again to the next launch: a
// batch's scans and folds rewrite the same sums and rows, so a repeat gives
// the same result.
constexpr int kRing = kDepth;
constexpr uint32_t kFinPerTicket = 256;
enum : uint32_t { kExitNone = 0, kExitIdle = 1, kExitStop = 2, kExitTimeout = 3 };
constexpr uint64_t kMaxWaitNs = 60ull * 1000000000ull; // the longest any one warp waits for its ticket
constexpr uint64_t kDrainStallNs = 2000000ull;           // a fold gives up after the spans stall this long
                                                         // while the kernel drains

struct BatchDesc {                 // host-written
    uint64_t seq;                  // batch number, from 1 (0: slot unused)
    uint64_t ticket0;              // first ticket
    uint32_t nSingle, nJoint, nFin, nFinTickets;
    const WorkItem *single, *joint;
    const FinItem *fin;
    const TableView *sv;
    const panel::View *jv;
    SegStats *sums;
};
constexpr int kDescWords = sizeof(BatchDesc) / 8;
static_assert(sizeof(BatchDesc) % 8 == 0 && kDescWords <= 32, "descriptor read by one warp, a word per lane");

struct Ctrl {                      // pinned host memory, written by the host
    uint64_t published;            // tickets published so far (release-stored)
    uint32_t stop, pad;
    BatchDesc slot[kRing];
};

struct Status {                    // pinned host memory, written by the kernel
    uint64_t doneSeq[kRing];       // last batch completed in each slot
    uint64_t tFirst[kRing], tDone[kRing]; // global timer (ns) of a batch's first claim and its completion
    uint32_t exitReason, pad;
    unsigned long long lookupFailures; // published tickets whose batch descriptor was not found
    unsigned long long foldGiveups;    // folds that gave up on stalled spans while the launch drained
};

struct DevState {                  // device memory, zeroed before each launch
    unsigned long long ticket;
    unsigned long long scanDone[kRing], finDone[kRing];
    unsigned long long published;  // device copy of the host's count (one warp at a time reads the host's)
    unsigned int draining;
    unsigned int polling;          // held by the warp reading the host's control block
    unsigned int stop;             // device copy of the host's stop flag
    unsigned long long lastGrowNs; // global time at which the poller last saw the count grow
    unsigned long long lastWorkNs; // global time at which a warp last finished a ticket
    BatchDesc desc[kRing];         // device copy of the ring's descriptors (seq 0 while rewritten)
};



__device__ __forceinline__ uint64_t ld_acquire_sys(const uint64_t *p)
{
    uint64_t v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_sys(uint64_t *p, uint64_t v)
{
    asm volatile("st.release.sys.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The published ticket count as this warp may rely on it: the device copy,
// refreshed (with the stop flag) from pinned host memory by one warp at a
// time. Waiting warps read only device memory: a whole grid polling the host
// would flood the host link, slowing the very uploads it waits for.
__device__ __forceinline__ uint64_t published_count(const Ctrl *ctrl, DevState *ds)
{
    uint64_t v = *(volatile unsigned long long *)&ds->published;
    if (atomicCAS(&ds->polling, 0u, 1u) == 0u) {
        const uint64_t h = ld_acquire_sys(&ctrl->published);
        const uint32_t stop = *(volatile const uint32_t *)&ctrl->stop;
        __threadfence_system();
        if (h > v) {
            // new batches: copy the ring's descriptors into device memory
            // before the device count covers them. A host slot read while the
            // host rewrites it (seq 0 or changed between the two reads) holds
            // a batch not yet published and is left for a later copy
            for (int i = 0; i < kRing; ++i) {
                const uint64_t *src = reinterpret_cast<const uint64_t *>(&ctrl->slot[i]);
                uint64_t w[kDescWords];
                const uint64_t sq = ld_acquire_sys(src);
                for (int j = 1; j < kDescWords; ++j)
                    w[j] = *(const volatile uint64_t *)(src + j);
                asm volatile("fence.acq_rel.sys;" ::: "memory");
                const uint64_t sq2 = *(const volatile uint64_t *)src;
                uint64_t *dst = reinterpret_cast<uint64_t *>(&ds->desc[i]);
                if (!sq || sq != sq2 || *(volatile uint64_t *)dst == sq)
                    continue;
                *(volatile uint64_t *)dst = 0; // readers skip the slot while it changes
                __threadfence();
                for (int j = 1; j < kDescWords; ++j)
                    *(volatile uint64_t *)(dst + j) = w[j];
                __threadfence();
                *(volatile uint64_t *)dst = sq;
            }
            __threadfence();
            atomicMax(&ds->lastGrowNs, (unsigned long long)global_ns());
        }
        atomicMax(&ds->published, (unsigned long long)h);
        if (stop)
            atomicExch(&ds->stop, 1u);
        __threadfence();
        atomicExch(&ds->polling, 0u);
        v = h > v ? h : v;
    }
    return v;
}

template <int NB, uint32_t K>
__global__ void __launch_bounds__(256, 3) k_serve_persistent(const Ctrl *ctrl, Status *status, DevState *ds,
                                                             const uint64_t *__restrict__ seq,
                                                             const uint64_t *__restrict__ mask, int k,
                                                             ibs_window *rows, uint64_t idleNs, uint64_t waitNs)
{
    const uint32_t lane = threadIdx.x & 31;
    // this warp's copy of the batch it worked on last
    uint64_t dT0 = 0, dEnd = 0;
    uint32_t slot = 0;
    uint64_t word = 0; // lane i < kDescWords: word i of that batch's descriptor
    for (;;) {
        // claim the next ticket, unless the kernel is stopping
        unsigned long long t = 0;
        uint32_t go = 0;
        if (lane == 0) {
            if (!*(volatile unsigned int *)&ds->draining && !*(volatile unsigned int *)&ds->stop) {
                t = atomicAdd(&ds->ticket, 1ull);
                // wait (bounded) until it is published. The kernel is idle when
                // the count has not grown for idleNs (tickets far ahead of the
                // count wait through steady traffic); no single wait exceeds
                // kMaxWaitNs; the spin count bounds the idle stretch as well
                const uint64_t t0 = global_ns();
                uint64_t idleFrom = t0;
                for (uint64_t spin = 0;; ++spin) {
                    if (published_count(ctrl, ds) > t) {
                        go = 1;
                        break;
                    }
                    if (*(volatile unsigned int *)&ds->draining || *(volatile unsigned int *)&ds->stop)
                        break;
                    // idle: neither new work published nor any ticket finished
                    // (a long batch keeps the kernel busy, not idle). Another
                    // warp may stamp its work after `now` was read: the quiet
                    // time is then zero, not a wrapped difference
                    const uint64_t now = global_ns();
                    const uint64_t grew = *(volatile unsigned long long *)&ds->lastGrowNs;
                    const uint64_t worked = *(volatile unsigned long long *)&ds->lastWorkNs;
                    const uint64_t active = grew > worked ? grew : worked;
                    if (active > idleFrom) {
                        idleFrom = active;
                        spin = 0;
                    }
                    const uint64_t quietNs = now > idleFrom ? now - idleFrom : 0;
                    if (quietNs > idleNs || spin > (idleNs >> 8) + 1024 || now - t0 > kMaxWaitNs) {
                        if (atomicExch(&ds->draining, 1u) == 0u)
                            *(volatile uint32_t *)&status->exitReason = kExitIdle;
                        break;
                    }
                    __nanosleep(spin < 64 ? 256 : 2048);
                }
                // leaving: the ticket may have been published after the last
                // refresh of the device copy; the host's count decides, and
                // then the device copy (descriptors included) is refreshed
                if (!go && ld_acquire_sys(&ctrl->published) > t)
                    for (int a = 0; a < (1 << 16) && !go; ++a) {
                        if (published_count(ctrl, ds) > t)
                            go = 1;
                        else
                            __nanosleep(256);
                    }
            }
        }
        go = __shfl_sync(dev::FULL_MASK, go, 0);
        if (!go)
            return;
        t = __shfl_sync(dev::FULL_MASK, t, 0);
        if (t < dT0 || t >= dEnd) {
            // find the ticket's batch among the ring's descriptors: lane i
            // looks at slot i; a descriptor read while the host rewrites it
            // is read again (a bounded number of times)
            __threadfence_system();
            uint32_t hit = 0;
            uint64_t t0 = 0, n = 0;
            for (int attempt = 0; attempt < 4096 && !hit; ++attempt) {
                if (attempt)
                    __nanosleep(256);
                t0 = 0;
                n = 0;
                if (lane < kRing) {
                    // the device copy of slot `lane`: a slot being rewritten
                    // shows seq 0 or a different seq on the second read, and
                    // only a slot read whole counts
                    const volatile uint64_t *w = reinterpret_cast<const volatile uint64_t *>(&ds->desc[lane]);
                    const uint64_t sq = w[0];
                    __threadfence();
                    t0 = w[1];
                    const uint64_t c0 = w[2], c1 = w[3];
                    __threadfence();
                    const uint64_t sq2 = w[0];
                    n = (sq && sq == sq2) ? (c0 & 0xffffffffu) + (c0 >> 32) + (c1 >> 32) : 0; // scan + fold tickets
                }
                hit = __ballot_sync(dev::FULL_MASK, lane < kRing && n && t >= t0 && t < t0 + n);
            }
            if (!hit) { // published tickets always have a descriptor: stop rather than guess
                if (lane == 0) {
                    atomicExch(&ds->draining, 1u);
                    *(volatile uint32_t *)&status->exitReason = kExitTimeout;
                    atomicAdd_system(&status->lookupFailures, 1ull);
                }
                return;
            }
            slot = __ffs(hit) - 1;
            dT0 = __shfl_sync(dev::FULL_MASK, t0, slot);
            dEnd = dT0 + __shfl_sync(dev::FULL_MASK, n, slot);
            word = 0;
            __threadfence();
            if (lane < kDescWords) // a live batch's device slot does not change
                word = reinterpret_cast<const volatile uint64_t *>(&ds->desc[slot])[lane];
        }
        // the descriptor's fields, from the lanes holding them
        BatchDesc d;
        {
            uint64_t *dp = reinterpret_cast<uint64_t *>(&d);
#pragma unroll
            for (int i = 0; i < kDescWords; ++i)
                dp[i] = __shfl_sync(dev::FULL_MASK, word, i);
        }
        const uint64_t local = t - d.ticket0;
        const uint64_t nScan = (uint64_t)d.nSingle + d.nJoint;
        if (local == 0 && lane == 0)
            *(volatile uint64_t *)&status->tFirst[slot] = global_ns();
        if (local < nScan) {
            if (local < d.nSingle) {
                const WorkItem it = d.single[local];
                serve_single_item<NB, K>(it, d.sv[it.view], seq, mask, d.sums, lane);
            } else {
                const WorkItem it = d.joint[local - d.nSingle];
                serve_joint_item<NB, K>(it, d.jv[it.view], seq, mask, d.sums, lane);
            }
            __threadfence(); // every lane's summaries are visible before the count
            __syncwarp();
            if (lane == 0) {
                atomicAdd(&ds->scanDone[slot], 1ull);
                atomicMax(&ds->lastWorkNs, (unsigned long long)global_ns());
            }
            continue;
        }
        // a fold ticket: wait (bounded) for the batch's scans. While the
        // kernel drains, a scan ticket of this batch may have been given up
        // by a leaving warp: when the count stops moving for kDrainStallNs
        // the fold gives up too, and the host publishes the batch again to
        // the next launch
        uint32_t ready = 1;
        if (lane == 0) {
            const uint64_t t0 = global_ns();
            uint64_t seen = 0, movedAt = t0;
            for (uint64_t spin = 0;; ++spin) {
                const uint64_t doneNow = *(volatile unsigned long long *)&ds->scanDone[slot];
                if (doneNow >= nScan)
                    break;
                const uint64_t now = global_ns();
                if (doneNow != seen) {
                    seen = doneNow;
                    movedAt = now;
                }
                if (*(volatile unsigned int *)&ds->draining && now - movedAt > kDrainStallNs) {
                    ready = 0;
                    atomicAdd_system(&status->foldGiveups, 1ull);
                    break;
                }
                if (now - t0 > waitNs || spin > (waitNs >> 8) + 1024) {
                    ready = 0;
                    atomicExch(&ds->draining, 1u);
                    *(volatile uint32_t *)&status->exitReason = kExitTimeout;
                    break;
                }
                __nanosleep(256);
            }
        }
        ready = __shfl_sync(dev::FULL_MASK, ready, 0);
        if (!ready)
            return;
        __threadfence(); // the summaries counted above are read after the count
        const uint64_t f0 = (local - nScan) * kFinPerTicket;
        const uint64_t f1 = f0 + kFinPerTicket < d.nFin ? f0 + kFinPerTicket : (uint64_t)d.nFin;
        for (uint64_t f = f0 + lane; f < f1; f += 32)
            serve_fin_item(d.fin[f], d.sums, k, rows);
        __threadfence_system(); // every lane's rows reach host memory before the batch is stamped done
        __syncwarp();
        if (lane == 0) {
            atomicMax(&ds->lastWorkNs, (unsigned long long)global_ns());
            if (atomicAdd(&ds->finDone[slot], 1ull) + 1 == d.nFinTickets) {
                // the batch's last fold: its counters are free for the slot's next batch
                ds->scanDone[slot] = 0;
                ds->finDone[slot] = 0;
                __threadfence_system();
                *(volatile uint64_t *)&status->tDone[slot] = global_ns();
                st_release_sys(&status->doneSeq[slot], d.seq);
            }
        }
    }
}

// First-fit allocator of [offset, offset+size) ranges of a pool.
class RangeAlloc
{
  public:
    explicit RangeAlloc(uint64_t size) { free_[0] = size; }
    bool alloc(uint64_t n, uint64_t &off)
    {
        if (n == 0) {
            off = 0;
            return true;
        }
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                off = it->first;
                const uint64_t rest = it->second - n;
                free_.erase(it);
                if (rest)
                    free_[off + n] = rest;
                return true;
            }
        return false;
    }
    void release(uint64_t off, uint64_t n)
    {
        if (n == 0)
            return;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

  private:
    std::map<uint64_t, uint64_t> free_;
};

// A device table holding one sample (single) or several (joint).
struct Group {
    uint32_t id = 0;
    bool joint = false;
    uint32_t nSamples = 1;
    TableGeom geom{};
    uint64_t stashBuckets = 0;       // joint tables: stash buckets of two {code, mask} entries
    uint64_t bucketBytes = 0, stashBytes = 0;
    void *host = nullptr;            // pinned image: buckets, then stash
    uint8_t *dev = nullptr;          // resident copy (pool memory) or null
    cudaEvent_t loaded = nullptr;    // reload completion
    bool loading = false;
    double lastUse = 0;
    int inflight = 0;                // launches in flight that use the table
    uint64_t cursor = 0;             // sweep position (global window index)
    uint64_t bytes() const { return bucketBytes + stashBytes; }
    TableView single_view() const
    {
        return TableView{geom, reinterpret_cast<const uint4 *>(dev),
                         stashBytes ? reinterpret_cast<const uint64_t *>(dev + bucketBytes) : nullptr};
    }
    panel::View joint_view() const
    {
        return panel::View{geom, reinterpret_cast<const uint4 *>(dev),
                           reinterpret_cast<const ulonglong2 *>(dev + bucketBytes), stashBuckets};
    }
};

struct SampleRef {
    uint32_t group, bit;
};

struct Request {
    uint64_t id = 0;
    uint32_t sample = 0, contig = 0;
    uint64_t w0 = 0, nw = 0, g0 = 0; // g0: global index of the first window
    uint64_t positions = 0;
    double submitT = 0;
    std::vector<std::pair<uint64_t, uint64_t>> remaining; // global windows not yet planned
    uint64_t planned = 0, rowOff = 0;
};

// An iteration's batch. In the persistent mode its states run Copying
// (items on their way to the device) -> Published -> done (Idle); a batch
// that was published when the kernel stopped goes back to Copying and is
// published to the next launch.
enum class BatchState { Idle, Copying, Published };

struct Launch {
    std::vector<uint32_t> groups;       // groups used (claimed: inflight)
    std::vector<Request *> finishing;   // requests whose last windows ran here
    cudaEvent_t start = nullptr, stop = nullptr;
    cudaEvent_t copied = nullptr;       // persistent mode: the items reached the device
    BatchState state = BatchState::Idle;
    uint64_t seq = 0;                   // persistent mode: batch number
    uint32_t nSingle = 0, nJoint = 0, nFin = 0, replays = 0;
    WorkItem *hSingle = nullptr, *hJoint = nullptr, *dSingle = nullptr, *dJoint = nullptr;
    FinItem *hFin = nullptr, *dFin = nullptr;
    TableView *hSV = nullptr, *dSV = nullptr;
    panel::View *hJV = nullptr, *dJV = nullptr;
    SegStats *dSums = nullptr;
    uint64_t positions = 0;        // reference positions scanned
    uint64_t samplePositions = 0;  // positions x samples answered by those scans
    bool active = false;
};

} // namespace serve
} // namespace ibs

using namespace ibs;
using namespace ibs::serve;

struct ibs_server {
    int device = 0;
    ibs_reference *ref = nullptr;
    uint32_t W = 0, k = 0;
    uint64_t budget = 0, resident = 0;
    uint64_t itemCap = kSumCap;
    bool serial = false; // one request per launch
    uint32_t tableFormat = 0;   // single-sample tables built by the server (0: tuned default)
    double keysPerBucket = 0;
    std::vector<std::unique_ptr<Group>> groups;
    std::vector<SampleRef> samples;
    std::vector<uint64_t> contigWin0; // global index of each contig's first window; back() = total
    cudaStream_t comp = nullptr, side = nullptr;
    ibs_window *dRows = nullptr;
    ibs_window *hRows = nullptr; // pinned mirror of dRows
    RangeAlloc rowAlloc{kRowPool};
    Launch launches[kDepth];
    int nextLaunch = 0;
    int sms = 148;
    // the persistent launch (batched mode unless iteration_launches)
    bool persistent = false;
    cudaStream_t copy = nullptr;          // item uploads while the kernel runs
    Ctrl *ctrl = nullptr;                 // pinned, mapped
    Status *status = nullptr;             // pinned, mapped
    Ctrl *dCtrl = nullptr;
    Status *dStatus = nullptr;
    DevState *ds = nullptr;
    ibs_window *dRowsMapped = nullptr;    // device address of hRows
    cudaEvent_t kernelEnd = nullptr;
    bool kernelRunning = false;
    int persistentGrid = 0;
    uint64_t nextSeq = 1, published = 0;
    uint64_t idleNs = 100000000ull, waitNs = 10000000000ull;
    uint64_t busyLastEnd = 0;
    // request state
    std::mutex mu;
    std::condition_variable cv, doneCv;
    std::deque<std::unique_ptr<Request>> queue;  // submitted, not admitted
    std::list<std::unique_ptr<Request>> active;  // admitted
    std::deque<ibs_request_result> done;
    std::vector<double> latencies;
    uint64_t nextId = 1;
    bool stop = false;
    std::thread worker;
    ibs_server_stats st{};
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::string fatal;
    double now() const
    {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    // window x (global index): its contig's packed base offset plus the window's bounds
    void window(uint64_t x, uint64_t &base, uint32_t &nPos, int32_t &start, int32_t &end) const
    {
        const uint32_t c = (uint32_t)(std::upper_bound(contigWin0.begin(), contigWin0.end(), x) -
                                      contigWin0.begin()) - 1;
        const uint64_t j = (x - contigWin0[c]) * ((uint64_t)W - k);
        const uint64_t e = std::min<uint64_t>(j + W, ref->lens[c]);
        base = ref->baseOff[c] + j;
        nPos = e - j >= k ? (uint32_t)(e - j - k + 1) : 0;
        start = (int32_t)j;
        end = (int32_t)e;
    }
};

namespace {

bool table_ready(Group &g)
{
    if (!g.dev)
        return false;
    if (g.loading) {
        if (cudaEventQuery(g.loaded) != cudaSuccess)
            return false;
        g.loading = false;
    }
    return true;
}

// Pending work of the groups in one planning pass: whether a group has
// requests with windows left, and the submission time of its oldest one.
struct Demand {
    std::vector<char> busy;
    std::vector<double> oldest;
};

// A group whose requests wait for more than this behind newer work may
// evict a table that still has pending requests.
constexpr double kEvictSlack = 0.25;

// Makes g resident, evicting least-recently-used idle tables. Tables with
// pending requests are kept unless g's oldest request is older than all of
// theirs by kEvictSlack: resident work finishes before its table is swapped
// out (no thrashing when many requests arrive together), and a long wait
// still gets its turn. Evicts nothing when g cannot be made to fit.
ibs_status make_resident(ibs_server *s, Group &g, const Demand *dem = nullptr, double gOldest = 0)
{
    if (g.dev)
        return IBS_OK;
    // a finished reload makes its table evictable, whether or not a request
    // has looked at it since (tables loaded at registration included)
    for (auto &o : s->groups)
        if (o->dev && o->loading)
            table_ready(*o);
    if (s->resident + g.bytes() > s->budget) {
        const uint64_t need = s->resident + g.bytes() - s->budget;
        std::vector<Group *> cand;
        for (auto &o : s->groups) {
            if (!o->dev || o->inflight || o->loading || o.get() == &g)
                continue;
            const bool busy = dem && dem->busy[o->id];
            if (busy && !(dem->oldest[o->id] > gOldest + kEvictSlack))
                continue;
            cand.push_back(o.get());
        }
        std::sort(cand.begin(), cand.end(), [dem](const Group *x, const Group *y) {
            const bool bx = dem && dem->busy[x->id], by = dem && dem->busy[y->id];
            return bx != by ? !bx : x->lastUse < y->lastUse;
        });
        uint64_t freed = 0;
        size_t take = 0;
        while (take < cand.size() && freed < need)
            freed += cand[take++]->bytes();
        if (freed < need)
            return IBS_ERR_STATE; // wait for tables in use to finish
        for (size_t i = 0; i < take; ++i) {
            Group *victim = cand[i];
            IBS_CUDA(cudaFreeAsync(victim->dev, s->side), "table eviction");
            victim->dev = nullptr;
            s->resident -= victim->bytes();
            s->st.evictions++;
        }
    }
    IBS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&g.dev), g.bytes(), s->side), "table reload alloc");
    IBS_CUDA(cudaMemcpyAsync(g.dev, g.host, g.bytes(), cudaMemcpyHostToDevice, s->side), "table reload");
    IBS_CUDA(cudaEventRecord(g.loaded, s->side), "table reload event");
    g.loading = true;
    s->resident += g.bytes();
    s->st.reloads++;
    s->st.reload_bytes += g.bytes();
    return IBS_OK;
}

ibs_request_result result_of(const Request &r, ibs_status status, double t)
{
    ibs_request_result res{};
    res.request_id = r.id;
    res.sample = r.sample;
    res.contig = r.contig;
    res.first_window = r.w0;
    res.n_windows = status == IBS_OK ? r.nw : 0;
    res.status = status;
    res.submit_time = r.submitT;
    res.done_time = t;
    return res;
}

// Completes launch L: its finishing requests' rows move to their results.
// Bookkeeping of a finished launch or batch: its tables are released and
// its finishing requests' rows move to their results.
void complete(ibs_server *s, Launch &L)
{
    const double t = s->now();
    std::lock_guard<std::mutex> lock(s->mu);
    for (uint32_t g : L.groups)
        s->groups[g]->inflight--;
    s->st.scanned += L.positions;
    s->st.sample_probes += L.samplePositions;
    for (Request *r : L.finishing) {
        ibs_request_result res = result_of(*r, IBS_OK, t);
        res.rows = static_cast<ibs_window *>(malloc(std::max<uint64_t>(r->nw, 1) * sizeof(ibs_window)));
        memcpy(res.rows, s->hRows + r->rowOff, r->nw * sizeof(ibs_window));
        s->rowAlloc.release(r->rowOff, r->nw);
        s->latencies.push_back(t - r->submitT);
        s->st.completed++;
        s->st.probes += r->positions;
        s->done.push_back(res);
        s->active.remove_if([r](const std::unique_ptr<Request> &p) { return p.get() == r; });
    }
    L.finishing.clear();
    L.groups.clear();
    L.active = false;
    L.state = BatchState::Idle;
    s->doneCv.notify_all();
}

void set_fatal(ibs_server *s, const std::string &msg)
{
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->fatal.empty())
        s->fatal = msg;
    s->doneCv.notify_all();
}

// Launches the persistent kernel over fresh device state; tickets count
// from 0 again.
bool start_kernel(ibs_server *s)
{
    s->ctrl->stop = 0;
    s->status->exitReason = kExitNone;
    memset(s->ctrl->slot, 0, sizeof(s->ctrl->slot)); // no descriptor of the last launch's ticket space survives
    __atomic_store_n(&s->ctrl->published, 0ull, __ATOMIC_RELEASE);
    s->published = 0;
    std::atomic_thread_fence(std::memory_order_seq_cst);
    cudaError_t e = cudaMemsetAsync(s->ds, 0, sizeof(DevState), s->comp);
    if (e == cudaSuccess) {
        if (s->k == 25)
            k_serve_persistent<kServeNB, 25><<<s->persistentGrid, 256, 0, s->comp>>>(
                s->dCtrl, s->dStatus, s->ds, s->ref->dSeq, s->ref->dMask, (int)s->k, s->dRowsMapped, s->idleNs,
                s->waitNs);
        else if (s->k == 31)
            k_serve_persistent<kServeNB, 31><<<s->persistentGrid, 256, 0, s->comp>>>(
                s->dCtrl, s->dStatus, s->ds, s->ref->dSeq, s->ref->dMask, (int)s->k, s->dRowsMapped, s->idleNs,
                s->waitNs);
        else
            k_serve_persistent<kServeNB, 0><<<s->persistentGrid, 256, 0, s->comp>>>(
                s->dCtrl, s->dStatus, s->ds, s->ref->dSeq, s->ref->dMask, (int)s->k, s->dRowsMapped, s->idleNs,
                s->waitNs);
        IBS_LAUNCHED();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaEventRecord(s->kernelEnd, s->comp);
    if (e != cudaSuccess) {
        set_fatal(s, std::string("CUDA error in the persistent serving launch: ") + cudaGetErrorString(e));
        return false;
    }
    s->kernelRunning = true;
    s->st.persistent_launches++;
    return true;
}

// Publishes batch L to the running kernel: its descriptor into its ring
// slot, then the ticket count (release).
void publish(ibs_server *s, Launch &L, int slot)
{
    BatchDesc d{};
    d.seq = L.seq;
    d.ticket0 = s->published;
    d.nSingle = L.nSingle;
    d.nJoint = L.nJoint;
    d.nFin = L.nFin;
    d.nFinTickets = std::max<uint32_t>(1, (L.nFin + kFinPerTicket - 1) / kFinPerTicket);
    d.single = L.dSingle;
    d.joint = L.dJoint;
    d.fin = L.dFin;
    d.sv = L.dSV;
    d.jv = L.dJV;
    d.sums = L.dSums;
    // seq last: a warp reading the slot while it changes sees seq 0 or a
    // changed seq and ignores it (the slot's previous batch is done, so no
    // live ticket belongs to it)
    BatchDesc *dst = &s->ctrl->slot[slot];
    __atomic_store_n(&dst->seq, 0ull, __ATOMIC_SEQ_CST);
    std::atomic_thread_fence(std::memory_order_seq_cst);
    const uint64_t seqNo = d.seq;
    d.seq = 0;
    *dst = d;
    __atomic_store_n(&dst->seq, seqNo, __ATOMIC_RELEASE);
    s->published += (uint64_t)d.nSingle + d.nJoint + d.nFinTickets;
    __atomic_store_n(&s->ctrl->published, s->published, __ATOMIC_RELEASE);
    L.state = BatchState::Published;
}

// The persistent mode's housekeeping, called by the loop between
// iterations: notices a stopped kernel (its unfinished batches go back to
// be published again), completes batches the kernel stamped done, and
// publishes copied batches in order, launching the kernel when needed.
void pump(ibs_server *s)
{
    if (s->kernelRunning && cudaEventQuery(s->kernelEnd) == cudaSuccess) {
        s->kernelRunning = false;
        const uint32_t why = *(volatile uint32_t *)&s->status->exitReason;
        if (why == kExitIdle)
            s->st.idle_exits++;
        else if (why == kExitTimeout)
            s->st.wait_timeouts++;
        s->st.lookup_failures = *(volatile unsigned long long *)&s->status->lookupFailures;
        s->st.fold_giveups = *(volatile unsigned long long *)&s->status->foldGiveups;
    }
    // batches the kernel stamped done, completed in batch order: a request's
    // rows can come from several batches, and it completes with the last
    // one, so an earlier batch must be done before a later one completes
    for (;;) {
        Launch *first = nullptr;
        int slot = -1;
        for (int i = 0; i < kDepth; ++i) {
            Launch &L = s->launches[i];
            if (L.state == BatchState::Published && (!first || L.seq < first->seq)) {
                first = &L;
                slot = i;
            }
        }
        if (!first || __atomic_load_n(&s->status->doneSeq[slot], __ATOMIC_ACQUIRE) != first->seq)
            break;
        const uint64_t a = *(volatile uint64_t *)&s->status->tFirst[slot];
        const uint64_t b = *(volatile uint64_t *)&s->status->tDone[slot];
        const uint64_t from = std::max(a, s->busyLastEnd);
        if (b > from)
            s->st.busy_seconds += (b - from) * 1e-9;
        s->busyLastEnd = std::max(s->busyLastEnd, b);
        complete(s, *first);
    }
    // published to a kernel that stopped before finishing them: publish again
    if (!s->kernelRunning)
        for (int i = 0; i < kDepth; ++i) {
            Launch &L = s->launches[i];
            if (L.state != BatchState::Published ||
                __atomic_load_n(&s->status->doneSeq[i], __ATOMIC_ACQUIRE) == L.seq)
                continue;
            if (++L.replays > 3) {
                set_fatal(s, "serving: a batch did not finish in four persistent launches (device wait timeout)");
                return;
            }
            s->st.replays++;
            L.state = BatchState::Copying; // its items are on the device already
        }
    // publication in batch order
    for (;;) {
        Launch *next = nullptr;
        int slot = -1;
        for (int i = 0; i < kDepth; ++i) {
            Launch &L = s->launches[i];
            if (L.state == BatchState::Copying && (!next || L.seq < next->seq)) {
                next = &L;
                slot = i;
            }
        }
        if (!next || cudaEventQuery(next->copied) != cudaSuccess)
            break;
        if (!s->kernelRunning && !start_kernel(s))
            break;
        publish(s, *next, slot);
    }
}

// Waits until launch or batch L has finished and completes it.
void retire(ibs_server *s, Launch &L)
{
    if (!s->persistent) {
        if (!L.active)
            return;
        cudaEventSynchronize(L.stop);
        float ms = 0;
        if (cudaEventElapsedTime(&ms, L.start, L.stop) == cudaSuccess)
            s->st.busy_seconds += ms * 1e-3;
        complete(s, L);
        return;
    }
    const auto t0 = std::chrono::steady_clock::now();
    while (L.state != BatchState::Idle) {
        pump(s);
        if (L.state == BatchState::Idle)
            break;
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (!s->fatal.empty())
                break;
        }
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(120)) {
            set_fatal(s, "serving: a batch did not finish within 120 s");
            break;
        }
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    L.active = false;
}

// Removes [lo, hi) (inside one of its intervals) from r's remaining windows.
void take(Request &r, uint64_t lo, uint64_t hi)
{
    for (size_t i = 0; i < r.remaining.size(); ++i) {
        auto &iv = r.remaining[i];
        if (lo < iv.first || hi > iv.second)
            continue;
        const std::pair<uint64_t, uint64_t> left{iv.first, lo}, right{hi, iv.second};
        r.remaining.erase(r.remaining.begin() + i);
        if (right.second > right.first)
            r.remaining.insert(r.remaining.begin() + i, right);
        if (left.second > left.first)
            r.remaining.insert(r.remaining.begin() + i, left);
        r.planned += hi - lo;
        return;
    }
}

// Plan budget of one launch.
struct Budget {
    uint64_t sums, positions, fins, items;
};

struct Piece {
    uint64_t a, b;
    Request *r;
    uint32_t bit;
};

// Plans the next run of pending windows of group g from its sweep cursor
// (or from the start of the single request's remaining windows when
// `cursorOverride` is set) into launch L. `used` counts the launch's
// summary slots, positions, rows and work items so far; this group stops at
// `limit` (its share), except that its first window may use anything left
// under `cap`, so that every group with a resident table makes progress.
void plan_group(ibs_server *s, Launch &L, Group &g, uint32_t view, const std::vector<Request *> &reqs,
                const Budget &limit, const Budget &cap, Budget &used, uint32_t &nSingle, uint32_t &nJoint,
                uint32_t &nFin, bool cursorOverride)
{
    const uint64_t NW = s->contigWin0.back();
    std::vector<Piece> pieces;
    for (Request *r : reqs)
        for (auto &iv : r->remaining)
            pieces.push_back(Piece{iv.first, iv.second, r, s->samples[r->sample].bit});
    if (pieces.empty())
        return;
    uint64_t cursor = cursorOverride ? pieces.front().a : g.cursor;
    uint64_t x0 = ~0ull;
    for (auto &p : pieces)
        if (p.b > cursor)
            x0 = std::min(x0, std::max(p.a, cursor));
    if (x0 == ~0ull) { // nothing at or after the cursor: wrap around
        cursor = 0;
        for (auto &p : pieces)
            x0 = std::min(x0, p.a);
    }
    // masks and requester counts of windows [x0, x0 + span) from per-bit difference arrays
    const uint64_t span = std::min<uint64_t>(NW - x0, 1u << 16);
    const uint32_t nBits = g.joint ? g.nSamples : 1;
    std::vector<int32_t> diff((size_t)nBits * (span + 1), 0);
    for (auto &p : pieces) {
        const uint64_t lo = std::max(p.a, x0), hi = std::min(p.b, x0 + span);
        if (lo >= hi)
            continue;
        diff[(size_t)p.bit * (span + 1) + (lo - x0)]++;
        diff[(size_t)p.bit * (span + 1) + (hi - x0)]--;
    }
    std::vector<int32_t> run(nBits, 0);
    std::vector<uint32_t> maskOf, baseOf;
    std::vector<uint64_t> sumOf;
    uint64_t x1 = x0;
    for (uint64_t x = x0; x < x0 + span; ++x) {
        uint32_t m = 0, requesters = 0;
        for (uint32_t b = 0; b < nBits; ++b) {
            run[b] += diff[(size_t)b * (span + 1) + (x - x0)];
            if (run[b] > 0) {
                m |= 1u << b;
                requesters += (uint32_t)run[b];
            }
        }
        uint64_t base;
        uint32_t nPos;
        int32_t st, en;
        s->window(x, base, nPos, st, en);
        const uint64_t spans = (nPos + kSpanLen - 1) / kSpanLen;
        const uint64_t slots = m ? spans * __builtin_popcount(m) : 0;
        const uint64_t pos = m ? nPos : 0;
        const uint64_t items = m ? spans : 0;
        auto within = [&](const Budget &b) {
            return used.sums + slots <= b.sums && used.positions + pos <= b.positions &&
                   used.fins + requesters <= b.fins && used.items + items <= b.items;
        };
        if (!(within(limit) || (x == x0 && within(cap))))
            break;
        maskOf.push_back(m);
        sumOf.push_back(used.sums);
        if (m) {
            for (uint64_t sp = 0; sp < spans; ++sp) {
                WorkItem it;
                it.base = base;
                it.p0 = (uint32_t)(sp * kSpanLen);
                it.p1 = std::min<uint32_t>(it.p0 + kSpanLen, nPos);
                it.view = view;
                it.mask = g.joint ? m : 1u;
                it.out = used.sums + sp * __builtin_popcount(m);
                if (g.joint)
                    L.hJoint[nJoint++] = it;
                else
                    L.hSingle[nSingle++] = it;
            }
            used.sums += slots;
            used.positions += pos;
            used.items += items;
            used.fins += requesters;
            L.positions += pos;
            L.samplePositions += pos * (uint64_t)__builtin_popcount(m);
        }
        x1 = x + 1;
    }
    // rows: every piece's windows inside [x0, x1)
    for (auto &p : pieces) {
        const uint64_t lo = std::max(p.a, x0), hi = std::min(p.b, x1);
        if (lo >= hi)
            continue;
        for (uint64_t x = lo; x < hi; ++x) {
            const uint32_t m = maskOf[x - x0];
            uint64_t base;
            uint32_t nPos;
            FinItem &f = L.hFin[nFin++];
            s->window(x, base, nPos, f.start, f.end);
            f.nSpans = (nPos + kSpanLen - 1) / kSpanLen;
            f.stride = __builtin_popcount(m);
            f.sum = sumOf[x - x0] + __builtin_popcount(m & ((1u << p.bit) - 1u));
            f.row = p.r->rowOff + (x - p.r->g0);
        }
        take(*p.r, lo, hi);
        if (p.r->planned == p.r->nw)
            L.finishing.push_back(p.r);
    }
    if (!cursorOverride)
        g.cursor = x1 >= NW ? 0 : x1;
}

void fail_requests(ibs_server *s, const std::vector<Request *> &reqs, double t)
{
    for (Request *r : reqs) {
        ibs_request_result res = result_of(*r, IBS_ERR_CUDA, t);
        res.rows = static_cast<ibs_window *>(malloc(sizeof(ibs_window)));
        s->rowAlloc.release(r->rowOff, r->nw);
        s->st.completed++;
        s->st.failed++;
        s->done.push_back(res);
        s->active.remove_if([r](const std::unique_ptr<Request> &p) { return p.get() == r; });
    }
    if (!reqs.empty())
        s->doneCv.notify_all();
}

// One loop iteration: plans and enqueues a launch. Returns false when there
// was nothing to run.
bool iterate(ibs_server *s)
{
    Launch &L = s->launches[s->nextLaunch];
    retire(s, L); // its staging buffers are reused below
    uint32_t nSingle = 0, nJoint = 0, nFin = 0, nSV = 0, nJV = 0;
    L.positions = 0;
    L.samplePositions = 0;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        // admit queued requests while the row pool has room
        while (!s->queue.empty() && !(s->serial && !s->active.empty())) {
            Request *r = s->queue.front().get();
            uint64_t ro;
            if (!s->rowAlloc.alloc(r->nw, ro))
                break;
            r->rowOff = ro;
            s->active.push_back(std::move(s->queue.front()));
            s->queue.pop_front();
        }
        // pending windows per group (one request in serial mode)
        std::map<uint32_t, std::vector<Request *>> demand;
        for (auto &rp : s->active) {
            if (rp->remaining.empty())
                continue; // every window planned; its last launch is in flight
            demand[s->samples[rp->sample].group].push_back(rp.get());
            if (s->serial)
                break;
        }
        const double t = s->now();
        // groups in the order of their oldest pending request
        Demand dem;
        dem.busy.assign(s->groups.size(), 0);
        dem.oldest.assign(s->groups.size(), 0.0);
        std::vector<std::pair<double, uint32_t>> order;
        for (auto &d : demand) {
            double o = d.second.front()->submitT;
            for (Request *r : d.second)
                o = std::min(o, r->submitT);
            dem.busy[d.first] = 1;
            dem.oldest[d.first] = o;
            order.push_back({o, d.first});
        }
        std::sort(order.begin(), order.end());
        std::vector<uint32_t> ready;
        for (auto &od : order) {
            auto &d = *demand.find(od.second);
            Group &g = *s->groups[d.first];
            if (!g.dev) {
                const ibs_status rs = make_resident(s, g, &dem, od.first);
                if (rs == IBS_ERR_STATE)
                    continue; // every resident table is busy: retry after a retire
                if (rs != IBS_OK) {
                    // a table that is not resident has no launch in flight,
                    // so none of these requests' windows is on the device
                    cudaGetLastError();
                    fail_requests(s, d.second, t);
                    continue;
                }
            }
            if (!table_ready(g))
                continue;
            g.lastUse = t;
            g.inflight++; // claimed: making another table resident cannot evict it now
            L.groups.push_back(d.first);
            ready.push_back(d.first);
        }
        if (ready.empty())
            return false;
        const Budget cap{kSumCap, kPosCap, kFinCap, s->itemCap};
        Budget used{0, 0, 0, 0};
        for (size_t i = 0; i < ready.size(); ++i) {
            const uint32_t gi = ready[i];
            Group &g = *s->groups[gi];
            const uint64_t left = ready.size() - i; // fair share of what the groups before left over
            const Budget limit{used.sums + (cap.sums - used.sums) / left,
                               used.positions + (cap.positions - used.positions) / left,
                               used.fins + (cap.fins - used.fins) / left,
                               used.items + (cap.items - used.items) / left};
            uint32_t view;
            if (g.joint) {
                view = nJV;
                L.hJV[nJV++] = g.joint_view();
            } else {
                view = nSV;
                L.hSV[nSV++] = g.single_view();
            }
            plan_group(s, L, g, view, demand[gi], limit, cap, used, nSingle, nJoint, nFin, s->serial);
        }
    }
    if (s->persistent) {
        // the items go up on the copy stream; the batch is published to the
        // running kernel once they are there
        cudaStream_t cs = s->copy;
        if (nSV)
            cudaMemcpyAsync(L.dSV, L.hSV, nSV * sizeof(TableView), cudaMemcpyHostToDevice, cs);
        if (nJV)
            cudaMemcpyAsync(L.dJV, L.hJV, nJV * sizeof(panel::View), cudaMemcpyHostToDevice, cs);
        if (nSingle)
            cudaMemcpyAsync(L.dSingle, L.hSingle, nSingle * sizeof(WorkItem), cudaMemcpyHostToDevice, cs);
        if (nJoint)
            cudaMemcpyAsync(L.dJoint, L.hJoint, nJoint * sizeof(WorkItem), cudaMemcpyHostToDevice, cs);
        if (nFin)
            cudaMemcpyAsync(L.dFin, L.hFin, nFin * sizeof(FinItem), cudaMemcpyHostToDevice, cs);
        cudaEventRecord(L.copied, cs);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            set_fatal(s, std::string("CUDA error in serving upload: ") + cudaGetErrorString(e));
        L.nSingle = nSingle;
        L.nJoint = nJoint;
        L.nFin = nFin;
        L.replays = 0;
        L.seq = s->nextSeq++;
        L.state = BatchState::Copying;
        L.active = true;
        s->st.launches++;
        s->st.spans += nSingle + nJoint;
        s->nextLaunch = (s->nextLaunch + 1) % kDepth;
        pump(s);
        return true;
    }
    cudaStream_t st = s->comp;
    if (nSV)
        cudaMemcpyAsync(L.dSV, L.hSV, nSV * sizeof(TableView), cudaMemcpyHostToDevice, st);
    if (nJV)
        cudaMemcpyAsync(L.dJV, L.hJV, nJV * sizeof(panel::View), cudaMemcpyHostToDevice, st);
    if (nSingle)
        cudaMemcpyAsync(L.dSingle, L.hSingle, nSingle * sizeof(WorkItem), cudaMemcpyHostToDevice, st);
    if (nJoint)
        cudaMemcpyAsync(L.dJoint, L.hJoint, nJoint * sizeof(WorkItem), cudaMemcpyHostToDevice, st);
    if (nFin)
        cudaMemcpyAsync(L.dFin, L.hFin, nFin * sizeof(FinItem), cudaMemcpyHostToDevice, st);
    cudaEventRecord(L.start, st);
    if (nSingle) {
        const int grid = (int)std::min<uint64_t>((nSingle + 7) / 8, (uint64_t)s->sms * 8);
        if (s->k == 25)
            k_serve_single<kServeNB, 25><<<grid, 256, 0, st>>>(L.dSV, L.dSingle, nSingle, s->ref->dSeq,
                                                          s->ref->dMask, L.dSums);
        else if (s->k == 31)
            k_serve_single<kServeNB, 31><<<grid, 256, 0, st>>>(L.dSV, L.dSingle, nSingle, s->ref->dSeq,
                                                          s->ref->dMask, L.dSums);
        else
            k_serve_single<kServeNB, 0><<<grid, 256, 0, st>>>(L.dSV, L.dSingle, nSingle, s->ref->dSeq,
                                                         s->ref->dMask, L.dSums);
        IBS_LAUNCHED();
    }
    if (nJoint) {
        const int grid = (int)std::min<uint64_t>((nJoint + 7) / 8, (uint64_t)s->sms * 8);
        if (s->k == 25)
            k_serve_joint<kNB, 25><<<grid, 256, 0, st>>>(L.dJV, L.dJoint, nJoint, s->ref->dSeq, s->ref->dMask,
                                                         L.dSums);
        else if (s->k == 31)
            k_serve_joint<kNB, 31><<<grid, 256, 0, st>>>(L.dJV, L.dJoint, nJoint, s->ref->dSeq, s->ref->dMask,
                                                         L.dSums);
        else
            k_serve_joint<kNB, 0><<<grid, 256, 0, st>>>(L.dJV, L.dJoint, nJoint, s->ref->dSeq, s->ref->dMask,
                                                        L.dSums);
        IBS_LAUNCHED();
    }
    if (nFin) {
        const int grid = (int)std::min<uint64_t>((nFin + 255) / 256, (uint64_t)s->sms * 8);
        k_serve_finalize<<<grid, 256, 0, st>>>(L.dFin, nFin, L.dSums, (int)s->k, s->dRows);
        IBS_LAUNCHED();
    }
    for (Request *r : L.finishing)
        if (r->nw)
            cudaMemcpyAsync(s->hRows + r->rowOff, s->dRows + r->rowOff, r->nw * sizeof(ibs_window),
                            cudaMemcpyDeviceToHost, st);
    cudaEventRecord(L.stop, st);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->fatal = std::string("CUDA error in serving launch: ") + cudaGetErrorString(e);
    }
    s->st.launches++;
    s->st.spans += nSingle + nJoint;
    L.active = true;
    s->nextLaunch = (s->nextLaunch + 1) % kDepth;
    return true;
}

void loop(ibs_server *s)
{
    cudaSetDevice(s->device);
    for (;;) {
        {
            std::unique_lock<std::mutex> lock(s->mu);
            if (s->stop)
                break;
        }
        if (iterate(s))
            continue;
        if (s->persistent) {
            // nothing to plan: keep the running batches moving and wait
            // briefly for new requests (a request arriving now is published
            // next to the batches in flight)
            pump(s);
            bool any = false;
            for (auto &L : s->launches)
                any |= L.state != BatchState::Idle;
            std::unique_lock<std::mutex> lock(s->mu);
            s->cv.wait_for(lock, any ? std::chrono::microseconds(20) : std::chrono::microseconds(1000),
                           [&] { return s->stop || !s->queue.empty(); });
            continue;
        }
        // nothing runnable: finish what is in flight, then wait for work
        bool any = false;
        for (auto &L : s->launches)
            if (L.active) {
                retire(s, L);
                any = true;
            }
        if (any)
            continue;
        std::unique_lock<std::mutex> lock(s->mu);
        s->cv.wait_for(lock, std::chrono::milliseconds(1),
                       [&] { return s->stop || !s->queue.empty(); });
    }
    for (auto &L : s->launches)
        retire(s, L);
}

// Registers a device table (copied to a pinned host image) as a group of
// n samples; returns the first sample id.
ibs_status add_group(ibs_server *s, bool joint, uint32_t nSamples, const TableGeom &geom, uint64_t stashBuckets,
                     const void *dBuckets, const void *dStash, uint32_t *first, ibs_panel_table *release = nullptr)
{
    if (geom.k != s->k) {
        set_error("server: the table's k differs from the server's k");
        return IBS_ERR_ARG;
    }
    std::unique_ptr<Group> g(new Group);
    g->joint = joint;
    g->nSamples = nSamples;
    g->geom = geom;
    g->stashBuckets = stashBuckets;
    g->bucketBytes = geom.nBuckets * 32;
    g->stashBytes = (joint ? stashBuckets : geom.stashBuckets) * 32;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->groups.size() >= kMaxGroups || s->samples.size() + nSamples > kMaxGroups) {
            set_error("server: at most 4096 samples");
            return IBS_ERR_CAPACITY;
        }
        if (g->bytes() > s->budget) {
            set_error("server: this table is larger than the memory budget");
            return IBS_ERR_CAPACITY;
        }
    }
    IBS_CUDA(cudaMallocHost(&g->host, g->bytes()), "pinned table image");
    IBS_CUDA(cudaMemcpy(g->host, dBuckets, g->bucketBytes, cudaMemcpyDeviceToHost), "table image");
    if (g->stashBytes)
        IBS_CUDA(cudaMemcpy(static_cast<uint8_t *>(g->host) + g->bucketBytes, dStash, g->stashBytes,
                            cudaMemcpyDeviceToHost),
                 "table image");
    IBS_CUDA(cudaEventCreateWithFlags(&g->loaded, cudaEventDisableTiming), "event create");
    if (release)
        panel_release_table(release);
    std::lock_guard<std::mutex> lock(s->mu);
    g->id = (uint32_t)s->groups.size();
    *first = (uint32_t)s->samples.size();
    for (uint32_t b = 0; b < nSamples; ++b)
        s->samples.push_back(SampleRef{g->id, b});
    s->groups.push_back(std::move(g));
    Group &ref = *s->groups.back();
    if (s->resident + ref.bytes() <= s->budget) {
        // resident now if the device has room; otherwise on its first request
        if (make_resident(s, ref) == IBS_OK) {
            s->st.reloads--; // the first load is not a reload
            s->st.reload_bytes -= ref.bytes();
        } else {
            cudaGetLastError();
            clear_error();
        }
    }
    return IBS_OK;
}

} // namespace

extern "C" ibs_status ibs_server_create(ibs_reference *ref, uint32_t W, uint32_t k,
                                        const ibs_server_opts *opts, ibs_server **out)
{
    clear_error();
    if (!ref || !out || k == 0 || k > 32 || W <= k) {
        set_error("ibs_server_create: bad argument (W must exceed k, k <= 32)");
        return IBS_ERR_ARG;
    }
    *out = nullptr;
    std::unique_ptr<ibs_server> s(new ibs_server);
    s->device = ref->device;
    s->ref = ref;
    s->W = W;
    s->k = k;
    DeviceGuard guard(s->device);
    if (opts && opts->max_spans_per_launch)
        s->itemCap = std::min<uint64_t>(opts->max_spans_per_launch, kSumCap);
    s->serial = opts && opts->one_request_per_launch;
    if (opts) {
        s->tableFormat = opts->table_format;
        s->keysPerBucket = opts->keys_per_bucket;
        if (opts->idle_exit_us)
            s->idleNs = (uint64_t)opts->idle_exit_us * 1000;
    }
    s->persistent = !s->serial && !(opts && opts->iteration_launches);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
    size_t fr = 0, tot = 0;
    IBS_CUDA(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
    s->budget = (opts && opts->memory_budget) ? opts->memory_budget : (uint64_t)(fr * 0.8);
    cudaMemPool_t pool;
    IBS_CUDA(cudaDeviceGetDefaultMemPool(&pool, s->device), "mempool");
    uint64_t threshold = ~0ull;
    IBS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "mempool");
    IBS_CUDA(cudaStreamCreateWithFlags(&s->comp, cudaStreamNonBlocking), "stream create");
    IBS_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking), "stream create");
    IBS_CUDA(cudaMalloc(&s->dRows, kRowPool * sizeof(ibs_window)), "row pool");
    IBS_CUDA(cudaMallocHost(&s->hRows, kRowPool * sizeof(ibs_window)), "pinned row pool");
    IBS_CUDA(cudaHostGetDevicePointer(&s->dRowsMapped, s->hRows, 0), "mapped row pool");
    if (s->persistent) {
        IBS_CUDA(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking), "stream create");
        IBS_CUDA(cudaHostAlloc(&s->ctrl, sizeof(Ctrl), cudaHostAllocMapped), "persistent control block");
        IBS_CUDA(cudaHostAlloc(&s->status, sizeof(Status), cudaHostAllocMapped), "persistent status block");
        memset(s->ctrl, 0, sizeof(Ctrl));
        memset(s->status, 0, sizeof(Status));
        IBS_CUDA(cudaHostGetDevicePointer(&s->dCtrl, s->ctrl, 0), "mapped control block");
        IBS_CUDA(cudaHostGetDevicePointer(&s->dStatus, s->status, 0), "mapped status block");
        IBS_CUDA(cudaMalloc(&s->ds, sizeof(DevState)), "persistent state");
        IBS_CUDA(cudaEventCreateWithFlags(&s->kernelEnd, cudaEventDisableTiming), "event create");
        int perSm = 0;
        if (s->k == 25)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_serve_persistent<kServeNB, 25>, 256, 0);
        else if (s->k == 31)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_serve_persistent<kServeNB, 31>, 256, 0);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_serve_persistent<kServeNB, 0>, 256, 0);
        s->persistentGrid = s->sms * std::max(1, perSm);
    }
    for (auto &L : s->launches) {
        IBS_CUDA(cudaEventCreate(&L.start), "event create");
        IBS_CUDA(cudaEventCreate(&L.stop), "event create");
        IBS_CUDA(cudaEventCreateWithFlags(&L.copied, cudaEventDisableTiming), "event create");
        IBS_CUDA(cudaMallocHost(&L.hSingle, kSumCap * sizeof(WorkItem)), "pinned staging");
        IBS_CUDA(cudaMallocHost(&L.hJoint, kSumCap * sizeof(WorkItem)), "pinned staging");
        IBS_CUDA(cudaMallocHost(&L.hFin, kFinCap * sizeof(FinItem)), "pinned staging");
        IBS_CUDA(cudaMallocHost(&L.hSV, kMaxGroups * sizeof(TableView)), "pinned staging");
        IBS_CUDA(cudaMallocHost(&L.hJV, kMaxGroups * sizeof(panel::View)), "pinned staging");
        IBS_CUDA(cudaMalloc(&L.dSingle, kSumCap * sizeof(WorkItem)), "staging");
        IBS_CUDA(cudaMalloc(&L.dJoint, kSumCap * sizeof(WorkItem)), "staging");
        IBS_CUDA(cudaMalloc(&L.dFin, kFinCap * sizeof(FinItem)), "staging");
        IBS_CUDA(cudaMalloc(&L.dSV, kMaxGroups * sizeof(TableView)), "staging");
        IBS_CUDA(cudaMalloc(&L.dJV, kMaxGroups * sizeof(panel::View)), "staging");
        IBS_CUDA(cudaMalloc(&L.dSums, kSumCap * sizeof(SegStats)), "summary pool");
    }
    s->contigWin0.push_back(0);
    for (size_t c = 0; c < ref->lens.size(); ++c)
        s->contigWin0.push_back(s->contigWin0.back() + windows_in_contig(ref->lens[c], W, k));
    ibs_server *raw = s.get();
    s->worker = std::thread(loop, raw);
    *out = s.release();
    return IBS_OK;
}

extern "C" ibs_status ibs_server_add_sample_codes(ibs_server *s, const uint64_t *codes, uint64_t n,
                                                  int on_device, uint32_t *id)
{
    clear_error();
    if (!s || !id) {
        set_error("ibs_server_add_sample_codes: bad argument");
        return IBS_ERR_ARG;
    }
    ibs_table_opts o{};
    o.device = s->device;
    o.force_format = s->tableFormat;
    o.keys_per_bucket = s->keysPerBucket;
    ibs_table *t = nullptr;
    ibs_status st = ibs_table_from_codes(codes, n, s->k, on_device, &o, &t);
    if (st != IBS_OK)
        return st;
    DeviceGuard guard(s->device);
    st = add_group(s, false, 1, t->geom, 0, t->buckets, t->stash, id);
    ibs_close(t);
    return st;
}

extern "C" ibs_status ibs_server_add_sample_kmc(ibs_server *s, const char *prefix, uint32_t *id)
{
    clear_error();
    if (!s || !prefix || !id) {
        set_error("ibs_server_add_sample_kmc: bad argument");
        return IBS_ERR_ARG;
    }
    ibs_table_opts o{};
    o.device = s->device;
    o.force_format = s->tableFormat;
    o.keys_per_bucket = s->keysPerBucket;
    ibs_table *t = nullptr;
    ibs_status st = ibs_open(prefix, &o, &t);
    if (st != IBS_OK)
        return st;
    DeviceGuard guard(s->device);
    st = add_group(s, false, 1, t->geom, 0, t->buckets, t->stash, id);
    ibs_close(t);
    return st;
}

extern "C" ibs_status ibs_server_add_panel(ibs_server *s, ibs_panel_table *p, int release_panel,
                                           uint32_t *first_id)
{
    clear_error();
    if (!s || !p || !first_id) {
        set_error("ibs_server_add_panel: bad argument");
        return IBS_ERR_ARG;
    }
    if (p->nSamples == 0) {
        set_error("ibs_server_add_panel: the panel table holds no samples");
        return IBS_ERR_ARG;
    }
    if (p->device != s->device) {
        set_error("ibs_server_add_panel: the panel table is on another device");
        return IBS_ERR_ARG;
    }
    if (!p->buckets) {
        set_error("ibs_server_add_panel: the panel's table was already released");
        return IBS_ERR_STATE;
    }
    DeviceGuard guard(s->device);
    // the host image first; then, when asked, the panel's device copy goes
    // before the server uploads its own, so that one copy is on the device
    ibs_status st = add_group(s, true, p->nSamples, p->geom, p->stashBuckets, p->buckets, p->stash, first_id,
                              release_panel ? p : nullptr);
    return st;
}

extern "C" ibs_status ibs_server_submit(ibs_server *s, uint32_t sample, uint32_t contig,
                                        uint64_t first, uint64_t n, uint64_t *request_id)
{
    clear_error();
    if (!s) {
        set_error("ibs_server_submit: bad argument");
        return IBS_ERR_ARG;
    }
    std::unique_ptr<Request> r(new Request);
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (!s->fatal.empty()) {
            set_error(s->fatal);
            return IBS_ERR_CUDA;
        }
        if (sample >= s->samples.size() || contig + 1 >= s->contigWin0.size()) {
            set_error("ibs_server_submit: unknown sample or contig");
            return IBS_ERR_ARG;
        }
    }
    const uint64_t nwC = s->contigWin0[contig + 1] - s->contigWin0[contig];
    if (first > nwC || (first == nwC && nwC)) {
        set_error("ibs_server_submit: first window beyond the contig");
        return IBS_ERR_ARG;
    }
    if (n == 0 || first + n > nwC)
        n = nwC - first;
    if (n > kRowPool) {
        set_error("ibs_server_submit: request larger than the server's row pool (split it)");
        return IBS_ERR_CAPACITY;
    }
    if (((uint64_t)s->W + kSpanLen - 1) / kSpanLen * IBS_PANEL_MAX_SAMPLES > kSumCap) {
        set_error("ibs_server_submit: windows this long do not fit one launch");
        return IBS_ERR_CAPACITY;
    }
    r->sample = sample;
    r->contig = contig;
    r->w0 = first;
    r->nw = n;
    r->g0 = s->contigWin0[contig] + first;
    if (n)
        r->remaining.push_back({r->g0, r->g0 + n});
    for (uint64_t x = r->g0; x < r->g0 + n; ++x) {
        uint64_t base;
        uint32_t nPos;
        int32_t a, b;
        s->window(x, base, nPos, a, b);
        r->positions += nPos;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->nextId++;
    r->submitT = s->now();
    if (request_id)
        *request_id = r->id;
    s->st.submitted++;
    if (n == 0) { // an empty contig has no windows: done at once
        ibs_request_result res = result_of(*r, IBS_OK, r->submitT);
        res.rows = static_cast<ibs_window *>(malloc(sizeof(ibs_window)));
        s->latencies.push_back(0.0);
        s->st.completed++;
        s->done.push_back(res);
        s->doneCv.notify_all();
        return IBS_OK;
    }
    s->queue.push_back(std::move(r));
    s->cv.notify_all();
    return IBS_OK;
}

extern "C" ibs_status ibs_server_poll(ibs_server *s, ibs_request_result *out, uint32_t max,
                                      uint32_t *n_out, int timeout_ms)
{
    clear_error();
    if (!s || !n_out || (max && !out)) {
        set_error("ibs_server_poll: bad argument");
        return IBS_ERR_ARG;
    }
    std::unique_lock<std::mutex> lock(s->mu);
    if (timeout_ms != 0 && s->done.empty()) {
        auto pred = [&] { return !s->done.empty() || !s->fatal.empty(); };
        if (timeout_ms < 0)
            s->doneCv.wait(lock, pred);
        else
            s->doneCv.wait_for(lock, std::chrono::milliseconds(timeout_ms), pred);
    }
    uint32_t n = 0;
    while (n < max && !s->done.empty()) {
        out[n++] = s->done.front();
        s->done.pop_front();
    }
    *n_out = n;
    if (!n && !s->fatal.empty()) {
        set_error(s->fatal);
        return IBS_ERR_CUDA;
    }
    return IBS_OK;
}

extern "C" void ibs_server_release(ibs_server *, ibs_request_result *r)
{
    if (r && r->rows) {
        free(r->rows);
        r->rows = nullptr;
    }
}

static double percentile(std::vector<double> v, double q)
{
    if (v.empty())
        return 0;
    std::sort(v.begin(), v.end());
    const double pos = q * (v.size() - 1);
    const size_t i = (size_t)pos;
    const double f = pos - i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

extern "C" ibs_status ibs_server_stats_get(ibs_server *s, ibs_server_stats *out)
{
    clear_error();
    if (!s || !out) {
        set_error("ibs_server_stats_get: bad argument");
        return IBS_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->st;
    out->resident_bytes = s->resident;
    uint64_t n = 0;
    for (auto &g : s->groups)
        n += g->dev ? 1 : 0;
    out->resident_tables = n;
    out->latency_p50 = percentile(s->latencies, 0.50);
    out->latency_p99 = percentile(s->latencies, 0.99);
    out->latency_max = s->latencies.empty() ? 0 : *std::max_element(s->latencies.begin(), s->latencies.end());
    out->queued = s->queue.size();
    out->running = s->active.size();
    return IBS_OK;
}

extern "C" double ibs_server_now(ibs_server *s) { return s ? s->now() : 0.0; }

extern "C" void ibs_server_close(ibs_server *s)
{
    if (!s)
        return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable())
        s->worker.join();
    {
        DeviceGuard guard(s->device);
        if (s->ctrl) // the persistent kernel's waiting warps see the stop and return
            __atomic_store_n(&s->ctrl->stop, 1u, __ATOMIC_RELEASE);
        cudaStreamSynchronize(s->comp);
        cudaStreamSynchronize(s->side);
        for (auto &g : s->groups) {
            if (g->dev)
                cudaFreeAsync(g->dev, s->side);
            cudaFreeHost(g->host);
            cudaEventDestroy(g->loaded);
        }
        cudaStreamSynchronize(s->side);
        // hand the tables' pool memory back, so that later allocations see it
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess)
            cudaMemPoolTrimTo(pool, 0);
        for (auto &L : s->launches) {
            cudaEventDestroy(L.start);
            cudaEventDestroy(L.stop);
            cudaFreeHost(L.hSingle);
            cudaFreeHost(L.hJoint);
            cudaFreeHost(L.hFin);
            cudaFreeHost(L.hSV);
            cudaFreeHost(L.hJV);
            cudaFree(L.dSingle);
            cudaFree(L.dJoint);
            cudaFree(L.dFin);
            cudaFree(L.dSV);
            cudaFree(L.dJV);
            cudaFree(L.dSums);
        }
        cudaFree(s->dRows);
        cudaFreeHost(s->hRows);
        if (s->copy) {
            cudaStreamSynchronize(s->copy);
            cudaStreamDestroy(s->copy);
        }
        for (auto &L : s->launches)
            cudaEventDestroy(L.copied);
        cudaFreeHost(s->ctrl);
        cudaFreeHost(s->status);
        cudaFree(s->ds);
        if (s->kernelEnd)
            cudaEventDestroy(s->kernelEnd);
        cudaStreamDestroy(s->comp);
        cudaStreamDestroy(s->side);
    }
    for (auto &r : s->done)
        free(r.rows);
    delete s;
}
