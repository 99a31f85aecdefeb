// The serving loop: continuous batching of window-scan requests over
// resident sample tables.
//
// A request names a sample and a range of windows of one contig. Its work
// is the spans of those windows (up to kSpanLen positions of one window
// each). A background thread runs the loop: admit requests, make their
// tables resident (least-recently-used eviction under a byte budget, reload
// from a pinned host image on a side stream), then launch one span kernel
// carrying slices of every runnable request -- each a work item that names
// its table -- followed by a finalizer for the requests whose last spans ran.
// Up to two launches are in flight; a request submitted meanwhile joins the
// next one. Rows are the same windows' rows of a full scan of the sample.
//
// No device code waits on the host: each launch is a finite kernel over a
// finite work list, so nothing here can spin on the GPU.
#include "ibs_internal.cuh"
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
constexpr uint64_t kSumPool = 4ull << 20;  // span summaries (32 B each): 128 MiB
constexpr uint64_t kRowPool = 2ull << 20;  // rows (24 B each): 48 MiB
constexpr int kDepth = 2;                  // launches in flight

struct WorkItem {
    uint64_t base;   // packed base offset of the window's first base
    uint32_t p0, p1; // positions of the window
    uint32_t table;  // index into this launch's table views
    uint32_t pad;
    uint64_t out;    // summary slot
};

struct FinItem {
    uint64_t sum;    // first summary slot of the window
    uint32_t nSpans;
    int32_t start, end;
    uint32_t pad;
    uint64_t row;    // row slot
};

template <int NB>
__global__ void __launch_bounds__(256) k_serve_spans(const TableView *__restrict__ views,
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
        const TableView t = views[it.table];
        const uint32_t k = t.g.k;
        const uint64_t kmask = key_mask(2 * k);
        const uint64_t kbits = (1ull << k) - 1;
        const bool b8 = t.g.format == FMT_B8X32;
        SegStats acc = seg_empty();
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
                acc = seg_combine(acc, dev::block_stats(V, H, lane, (int)k), (int)k);
            }
        }
        if (lane == 0)
            sums[it.out] = acc;
    }
}

__global__ void k_serve_finalize(const FinItem *__restrict__ fin, uint32_t n, const SegStats *__restrict__ sums,
                                 int k, ibs_window *__restrict__ rows)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const FinItem f = fin[i];
        SegStats acc = seg_empty();
        for (uint32_t s = 0; s < f.nSpans; ++s)
            acc = seg_combine(acc, sums[f.sum + s], k);
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

struct Sample {
    uint32_t id = 0;
    TableGeom geom{};
    uint64_t nKeys = 0;
    uint64_t bucketBytes = 0, stashBytes = 0;
    void *host = nullptr;            // pinned image: buckets, then stash
    uint8_t *dev = nullptr;          // resident copy (pool memory) or null
    cudaEvent_t loaded = nullptr;    // reload completion
    bool loading = false;
    double lastUse = 0;
    int inflight = 0;                // launches in flight that use the table
    uint64_t bytes() const { return bucketBytes + stashBytes; }
    TableView view() const
    {
        return TableView{geom, reinterpret_cast<const uint4 *>(dev),
                         stashBytes ? reinterpret_cast<const uint64_t *>(dev + bucketBytes) : nullptr};
    }
};

struct Request {
    uint64_t id = 0;
    uint32_t sample = 0, contig = 0;
    uint64_t w0 = 0, nw = 0;
    double submitT = 0;
    std::vector<FinItem> win;        // per window (sum/row relative to the request's slots)
    std::vector<uint64_t> winBase;   // packed base per window
    std::vector<uint32_t> winPos;    // positions per window
    uint64_t totalSpans = 0, scheduled = 0;
    uint64_t sumOff = 0, rowOff = 0;
    uint64_t curWin = 0, curSpanInWin = 0; // scheduling cursor
    bool admitted = false;
};

struct Launch {
    std::vector<uint32_t> tables;       // sample ids used
    std::vector<Request *> finishing;   // requests whose last spans ran here
    cudaEvent_t start = nullptr, stop = nullptr;
    WorkItem *hItems = nullptr;
    FinItem *hFin = nullptr;
    TableView *hViews = nullptr;
    WorkItem *dItems = nullptr;
    FinItem *dFin = nullptr;
    TableView *dViews = nullptr;
    uint64_t probes = 0;
    uint32_t nItems = 0;
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
    uint32_t maxItems = 1u << 15, minPer = 16;
    bool serial = false; // one whole request per launch
    std::vector<std::unique_ptr<Sample>> samples;
    std::vector<std::vector<uint64_t>> contigWin; // per contig: window count
    cudaStream_t comp = nullptr, side = nullptr;
    SegStats *dSums = nullptr;
    ibs_window *dRows = nullptr;
    ibs_window *hRows = nullptr; // pinned mirror of dRows
    RangeAlloc sumAlloc{kSumPool}, rowAlloc{kRowPool};
    Launch launches[kDepth];
    int nextLaunch = 0;
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
};

namespace {

bool table_ready(Sample &smp);

ibs_status make_resident(ibs_server *s, Sample &smp)
{
    if (smp.dev)
        return IBS_OK;
    // a finished reload makes its table evictable, whether or not a request
    // has looked at it since (tables loaded at registration included)
    for (auto &o : s->samples)
        if (o->dev && o->loading)
            table_ready(*o);
    // evict least-recently-used idle tables until this one fits
    while (s->resident + smp.bytes() > s->budget) {
        Sample *victim = nullptr;
        for (auto &o : s->samples)
            if (o->dev && !o->inflight && !o->loading && (!victim || o->lastUse < victim->lastUse))
                victim = o.get();
        if (!victim)
            return IBS_ERR_STATE; // everything resident is in use: retry later
        IBS_CUDA(cudaFreeAsync(victim->dev, s->side), "table eviction");
        victim->dev = nullptr;
        s->resident -= victim->bytes();
        s->st.evictions++;
    }
    IBS_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&smp.dev), smp.bytes(), s->side), "table reload alloc");
    IBS_CUDA(cudaMemcpyAsync(smp.dev, smp.host, smp.bytes(), cudaMemcpyHostToDevice, s->side), "table reload");
    IBS_CUDA(cudaEventRecord(smp.loaded, s->side), "table reload event");
    smp.loading = true;
    s->resident += smp.bytes();
    s->st.reloads++;
    s->st.reload_bytes += smp.bytes();
    return IBS_OK;
}

bool table_ready(Sample &smp)
{
    if (!smp.dev)
        return false;
    if (smp.loading) {
        if (cudaEventQuery(smp.loaded) != cudaSuccess)
            return false;
        smp.loading = false;
    }
    return true;
}

// Completes launch L: its finishing requests' rows move to their results.
void retire(ibs_server *s, Launch &L)
{
    if (!L.active)
        return;
    cudaEventSynchronize(L.stop);
    float ms = 0;
    if (cudaEventElapsedTime(&ms, L.start, L.stop) == cudaSuccess)
        s->st.busy_seconds += ms * 1e-3;
    const double t = s->now();
    std::lock_guard<std::mutex> lock(s->mu);
    for (uint32_t id : L.tables)
        s->samples[id]->inflight--;
    s->st.probes += L.probes;
    for (Request *r : L.finishing) {
        ibs_request_result res{};
        res.request_id = r->id;
        res.sample = r->sample;
        res.contig = r->contig;
        res.first_window = r->w0;
        res.n_windows = r->nw;
        res.status = IBS_OK;
        res.submit_time = r->submitT;
        res.done_time = t;
        res.rows = static_cast<ibs_window *>(malloc(std::max<uint64_t>(r->nw, 1) * sizeof(ibs_window)));
        memcpy(res.rows, s->hRows + r->rowOff, r->nw * sizeof(ibs_window));
        s->sumAlloc.release(r->sumOff, r->totalSpans);
        s->rowAlloc.release(r->rowOff, r->nw);
        s->latencies.push_back(t - r->submitT);
        s->st.completed++;
        s->done.push_back(res);
        for (auto it = s->active.begin(); it != s->active.end(); ++it)
            if (it->get() == r) {
                s->active.erase(it);
                break;
            }
    }
    L.finishing.clear();
    L.tables.clear();
    L.active = false;
    s->doneCv.notify_all();
}

// One loop iteration: plans and enqueues a launch. Returns false when there
// was nothing to run.
bool iterate(ibs_server *s)
{
    Launch &L = s->launches[s->nextLaunch];
    retire(s, L); // its staging buffers are reused below
    std::vector<Request *> runnable;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        // admit queued requests while the summary and row pools have room
        while (!s->queue.empty() && !(s->serial && !s->active.empty())) {
            Request *r = s->queue.front().get();
            uint64_t so, ro;
            if (!s->sumAlloc.alloc(r->totalSpans, so))
                break;
            if (!s->rowAlloc.alloc(r->nw, ro)) {
                s->sumAlloc.release(so, r->totalSpans);
                break;
            }
            r->sumOff = so;
            r->rowOff = ro;
            for (auto &f : r->win) {
                f.sum += so;
                f.row += ro;
            }
            r->admitted = true;
            s->active.push_back(std::move(s->queue.front()));
            s->queue.pop_front();
        }
        const double t = s->now();
        std::vector<Request *> failed;
        for (auto &rp : s->active) {
            Request *r = rp.get();
            if (r->curWin == r->nw)
                continue; // every span issued; its finalize is in flight
            Sample &smp = *s->samples[r->sample];
            if (!smp.dev) {
                const ibs_status rs = make_resident(s, smp);
                if (rs == IBS_ERR_STATE)
                    continue; // every resident table is busy: retry after a retire
                if (rs != IBS_OK) {
                    // a table that is not resident has no launch in flight,
                    // so none of this request's spans is on the device
                    cudaGetLastError();
                    failed.push_back(r);
                    continue;
                }
            }
            if (!table_ready(smp))
                continue;
            smp.lastUse = t;
            // claim the table for this launch now, so that making another
            // request's table resident cannot evict it while we plan
            if (std::find(L.tables.begin(), L.tables.end(), r->sample) == L.tables.end()) {
                smp.inflight++;
                L.tables.push_back(r->sample);
            }
            runnable.push_back(r);
        }
        for (Request *r : failed) {
            ibs_request_result res{};
            res.request_id = r->id;
            res.sample = r->sample;
            res.contig = r->contig;
            res.first_window = r->w0;
            res.n_windows = 0;
            res.status = IBS_ERR_CUDA;
            res.submit_time = r->submitT;
            res.done_time = t;
            res.rows = static_cast<ibs_window *>(malloc(sizeof(ibs_window)));
            s->sumAlloc.release(r->sumOff, r->totalSpans);
            s->rowAlloc.release(r->rowOff, r->nw);
            s->st.completed++;
            s->st.failed++;
            s->done.push_back(res);
            s->active.remove_if([r](const std::unique_ptr<Request> &p) { return p.get() == r; });
        }
        if (!failed.empty())
            s->doneCv.notify_all();
    }
    if (runnable.empty()) {
        std::lock_guard<std::mutex> lock(s->mu);
        for (uint32_t id : L.tables)
            s->samples[id]->inflight--;
        L.tables.clear();
        return false;
    }
    // spans: every runnable request gets a share of the launch
    const uint64_t share =
        s->serial ? ~0ull : std::max<uint64_t>(s->minPer, s->maxItems / runnable.size());
    uint32_t nItems = 0, nFin = 0;
    std::map<uint32_t, uint32_t> slot; // sample -> view index
    L.probes = 0;
    for (uint32_t i = 0; i < L.tables.size(); ++i) {
        slot[L.tables[i]] = i;
        L.hViews[i] = s->samples[L.tables[i]]->view();
    }
    for (Request *r : runnable) {
        const uint32_t vi = slot[r->sample];
        uint64_t taken = 0;
        while (r->curWin < r->nw && taken < share && nItems < s->maxItems) {
            const uint32_t nPos = r->winPos[r->curWin];
            const uint64_t spans = (nPos + kSpanLen - 1) / kSpanLen;
            if (r->curSpanInWin < spans) {
                WorkItem &it = L.hItems[nItems++];
                it.base = r->winBase[r->curWin];
                it.p0 = (uint32_t)(r->curSpanInWin * kSpanLen);
                it.p1 = std::min<uint32_t>(it.p0 + kSpanLen, nPos);
                it.table = vi;
                it.pad = 0;
                it.out = r->win[r->curWin].sum + r->curSpanInWin;
                L.probes += it.p1 - it.p0;
                r->curSpanInWin++;
                r->scheduled++;
                taken++;
            }
            if (r->curSpanInWin >= spans) {
                r->curWin++;
                r->curSpanInWin = 0;
            }
        }
        if (r->curWin == r->nw) { // last spans issued: finalize in this launch
            for (uint64_t w = 0; w < r->nw; ++w)
                L.hFin[nFin++] = r->win[w];
            L.finishing.push_back(r);
        }
        if (nItems >= s->maxItems)
            break;
    }
    L.nItems = nItems;
    cudaStream_t st = s->comp;
    cudaMemcpyAsync(L.dViews, L.hViews, slot.size() * sizeof(TableView), cudaMemcpyHostToDevice, st);
    if (nItems)
        cudaMemcpyAsync(L.dItems, L.hItems, nItems * sizeof(WorkItem), cudaMemcpyHostToDevice, st);
    if (nFin)
        cudaMemcpyAsync(L.dFin, L.hFin, nFin * sizeof(FinItem), cudaMemcpyHostToDevice, st);
    cudaEventRecord(L.start, st);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (nItems) {
        const int grid = (int)std::min<uint64_t>((nItems + 7) / 8, (uint64_t)sms * 8);
        k_serve_spans<kNB><<<grid, 256, 0, st>>>(L.dViews, L.dItems, nItems, s->ref->dSeq, s->ref->dMask,
                                                 s->dSums);
        IBS_LAUNCHED();
    }
    cudaEventRecord(L.stop, st);
    if (nFin) {
        const int grid = (int)std::min<uint64_t>((nFin + 255) / 256, (uint64_t)sms * 8);
        k_serve_finalize<<<grid, 256, 0, st>>>(L.dFin, nFin, s->dSums, (int)s->k, s->dRows);
        IBS_LAUNCHED();
        for (Request *r : L.finishing)
            if (r->nw)
                cudaMemcpyAsync(s->hRows + r->rowOff, s->dRows + r->rowOff, r->nw * sizeof(ibs_window),
                                cudaMemcpyDeviceToHost, st);
        cudaEventRecord(L.stop, st); // results ready
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lock(s->mu);
        s->fatal = std::string("CUDA error in serving launch: ") + cudaGetErrorString(e);
    }
    s->st.launches++;
    s->st.spans += nItems;
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

ibs_status add_table(ibs_server *s, ibs_table *t, uint32_t *id)
{
    std::unique_ptr<Sample> smp(new Sample);
    smp->geom = t->geom;
    smp->nKeys = t->nKeys;
    smp->bucketBytes = t->geom.nBuckets * 32;
    smp->stashBytes = t->geom.stashBuckets * 32;
    IBS_CUDA(cudaMallocHost(&smp->host, smp->bytes()), "pinned table image");
    IBS_CUDA(cudaMemcpy(smp->host, t->buckets, smp->bucketBytes, cudaMemcpyDeviceToHost), "table image");
    if (smp->stashBytes)
        IBS_CUDA(cudaMemcpy(static_cast<uint8_t *>(smp->host) + smp->bucketBytes, t->stash, smp->stashBytes,
                            cudaMemcpyDeviceToHost),
                 "table image");
    IBS_CUDA(cudaEventCreateWithFlags(&smp->loaded, cudaEventDisableTiming), "event create");
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->samples.size() >= 4096) {
        set_error("server: at most 4096 samples");
        return IBS_ERR_CAPACITY;
    }
    if (smp->bytes() > s->budget) {
        set_error("server: this sample's table is larger than the memory budget");
        return IBS_ERR_CAPACITY;
    }
    if (t->geom.k != s->k) {
        set_error("server: sample k differs from the server's k");
        return IBS_ERR_ARG;
    }
    smp->id = (uint32_t)s->samples.size();
    *id = smp->id;
    s->samples.push_back(std::move(smp));
    Sample &ref = *s->samples.back();
    if (s->resident + ref.bytes() <= s->budget) {
        ibs_status st = make_resident(s, ref);
        if (st != IBS_OK)
            return st;
        s->st.reloads--; // the first load is not a reload
        s->st.reload_bytes -= ref.bytes();
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
        s->maxItems = opts->max_spans_per_launch;
    if (opts && opts->min_spans_per_request)
        s->minPer = opts->min_spans_per_request;
    s->serial = opts && opts->one_request_per_launch;
    if (s->serial)
        s->maxItems = std::max<uint32_t>(s->maxItems, (uint32_t)kSumPool);
    size_t fr = 0, tot = 0;
    IBS_CUDA(cudaMemGetInfo(&fr, &tot), "cudaMemGetInfo");
    s->budget = (opts && opts->memory_budget) ? opts->memory_budget : (uint64_t)(fr * 0.8);
    cudaMemPool_t pool;
    IBS_CUDA(cudaDeviceGetDefaultMemPool(&pool, s->device), "mempool");
    uint64_t threshold = ~0ull;
    IBS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold), "mempool");
    IBS_CUDA(cudaStreamCreateWithFlags(&s->comp, cudaStreamNonBlocking), "stream create");
    IBS_CUDA(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking), "stream create");
    IBS_CUDA(cudaMalloc(&s->dSums, kSumPool * sizeof(SegStats)), "summary pool");
    IBS_CUDA(cudaMalloc(&s->dRows, kRowPool * sizeof(ibs_window)), "row pool");
    IBS_CUDA(cudaMallocHost(&s->hRows, kRowPool * sizeof(ibs_window)), "pinned row pool");
    for (auto &L : s->launches) {
        IBS_CUDA(cudaEventCreate(&L.start), "event create");
        IBS_CUDA(cudaEventCreate(&L.stop), "event create");
        IBS_CUDA(cudaMallocHost(&L.hItems, s->maxItems * sizeof(WorkItem)), "pinned staging");
        IBS_CUDA(cudaMallocHost(&L.hFin, kRowPool * sizeof(FinItem)), "pinned staging");
        IBS_CUDA(cudaMallocHost(&L.hViews, 4096 * sizeof(TableView)), "pinned staging");
        IBS_CUDA(cudaMalloc(&L.dItems, s->maxItems * sizeof(WorkItem)), "staging");
        IBS_CUDA(cudaMalloc(&L.dFin, kRowPool * sizeof(FinItem)), "staging");
        IBS_CUDA(cudaMalloc(&L.dViews, 4096 * sizeof(TableView)), "staging");
    }
    for (size_t c = 0; c < ref->lens.size(); ++c)
        s->contigWin.push_back({windows_in_contig(ref->lens[c], W, k)});
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
    o.force_format = FMT_AUTO_HASH; // the serving kernel probes the hash-bucket formats
    ibs_table *t = nullptr;
    ibs_status st = ibs_table_from_codes(codes, n, s->k, on_device, &o, &t);
    if (st != IBS_OK)
        return st;
    DeviceGuard guard(s->device);
    st = add_table(s, t, id);
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
    o.force_format = FMT_AUTO_HASH;
    ibs_table *t = nullptr;
    ibs_status st = ibs_open(prefix, &o, &t);
    if (st != IBS_OK)
        return st;
    DeviceGuard guard(s->device);
    st = add_table(s, t, id);
    ibs_close(t);
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
        if (sample >= s->samples.size() || contig >= s->contigWin.size()) {
            set_error("ibs_server_submit: unknown sample or contig");
            return IBS_ERR_ARG;
        }
    }
    const uint64_t nwC = s->contigWin[contig][0];
    if (first > nwC || (first == nwC && nwC)) {
        set_error("ibs_server_submit: first window beyond the contig");
        return IBS_ERR_ARG;
    }
    if (n == 0 || first + n > nwC)
        n = nwC - first;
    r->sample = sample;
    r->contig = contig;
    r->w0 = first;
    r->nw = n;
    const uint64_t L = s->ref->lens[contig];
    const uint64_t step = (uint64_t)s->W - s->k;
    uint64_t spans = 0;
    r->win.resize(n);
    r->winBase.resize(n);
    r->winPos.resize(n);
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t j = (first + i) * step;
        const uint64_t end = std::min<uint64_t>(j + s->W, L);
        const uint64_t nb = end - j;
        const uint32_t nPos = nb >= s->k ? (uint32_t)(nb - s->k + 1) : 0;
        FinItem &f = r->win[i];
        f.sum = spans;
        f.nSpans = (nPos + kSpanLen - 1) / kSpanLen;
        f.start = (int32_t)j;
        f.end = (int32_t)end;
        f.pad = 0;
        f.row = i;
        r->winBase[i] = s->ref->baseOff[contig] + j;
        r->winPos[i] = nPos;
        spans += f.nSpans;
    }
    r->totalSpans = spans;
    if (spans > kSumPool || n > kRowPool) {
        set_error("ibs_server_submit: request larger than the server's pools (split it)");
        return IBS_ERR_CAPACITY;
    }
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->nextId++;
    r->submitT = s->now();
    if (request_id)
        *request_id = r->id;
    s->st.submitted++;
    if (n == 0) { // an empty contig has no windows: done at once
        ibs_request_result res{};
        res.request_id = r->id;
        res.sample = sample;
        res.contig = contig;
        res.first_window = first;
        res.status = IBS_OK;
        res.submit_time = res.done_time = r->submitT;
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
    for (auto &smp : s->samples)
        n += smp->dev ? 1 : 0;
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
        cudaStreamSynchronize(s->comp);
        cudaStreamSynchronize(s->side);
        for (auto &smp : s->samples) {
            if (smp->dev)
                cudaFreeAsync(smp->dev, s->side);
            cudaFreeHost(smp->host);
            cudaEventDestroy(smp->loaded);
        }
        cudaStreamSynchronize(s->side);
        for (auto &L : s->launches) {
            cudaEventDestroy(L.start);
            cudaEventDestroy(L.stop);
            cudaFreeHost(L.hItems);
            cudaFreeHost(L.hFin);
            cudaFreeHost(L.hViews);
            cudaFree(L.dItems);
            cudaFree(L.dFin);
            cudaFree(L.dViews);
        }
        cudaFree(s->dSums);
        cudaFree(s->dRows);
        cudaFreeHost(s->hRows);
        cudaStreamDestroy(s->comp);
        cudaStreamDestroy(s->side);
    }
    for (auto &r : s->done)
        free(r.rows);
    delete s;
}
