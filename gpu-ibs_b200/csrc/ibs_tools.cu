// libibs_tools: seeded synthetic references/samples and a KMC 3 writer.
// Test and benchmark infrastructure: the scan library does not link it.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ibs_tools.h"
#include "ibs_core.cuh"
#include "synth_core.cuh"

using namespace ibs;
using namespace ibs::synth;

namespace {

thread_local std::string g_err;

ibs_status fail(ibs_status s, const std::string &m)
{
    g_err = m;
    return s;
}

#define TCUDA(call, what)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            cudaGetLastError();                                                                \
            return fail(e_ == cudaErrorMemoryAllocation ? IBS_ERR_NOMEM : IBS_ERR_CUDA,        \
                        std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e_)); \
        }                                                                                      \
    } while (0)

int hw_threads() { return (int)std::max(1u, std::thread::hardware_concurrency()); }

template <typename F> void parallel_for(uint64_t n, int threads, F f)
{
    threads = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)threads, n));
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        for (uint64_t i; (i = next.fetch_add(1)) < n;)
            f(i);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t)
        pool.emplace_back(work);
    work();
    for (auto &th : pool)
        th.join();
}

struct Run {
    uint32_t c;
    uint64_t start, len;
};

std::vector<Run> make_runs(const ibs_synth_ref_spec *s, uint64_t streamBase, double frac,
                           uint32_t rmin, uint32_t rmax)
{
    std::vector<Run> runs;
    if (frac <= 0 || rmax < rmin || rmax == 0)
        return runs;
    const double mean = (rmin + rmax) / 2.0;
    for (uint32_t c = 0; c < s->n_contigs; ++c) {
        const uint64_t len = s->lens[c];
        if (!len)
            continue;
        const uint64_t n = (uint64_t)((double)len * frac / mean);
        for (uint64_t r = 0; r < n; ++r) {
            const uint64_t st = rnd(s->seed, streamBase + c, 2 * r) % len;
            const uint64_t ln = rmin + rnd(s->seed, streamBase + c, 2 * r + 1) % (rmax - rmin + 1);
            runs.push_back({c, st, std::min(ln, len - st)});
        }
    }
    return runs;
}

void offsets(const ibs_synth_ref_spec *s, std::vector<uint64_t> &off, uint64_t &seqWords,
             uint64_t &maskWords)
{
    off.resize(s->n_contigs);
    uint64_t b = 0;
    for (uint32_t c = 0; c < s->n_contigs; ++c) {
        off[c] = b;
        b += round_up64(s->lens[c]);
    }
    seqWords = b / 32 + 1;
    maskWords = b / 64 + 1;
}

// 32 mask bits (one per base) -> 64-bit mask of the bases' 2-bit fields.
IBS_HD uint64_t spread2(uint32_t m)
{
    uint64_t x = m;
    x = (x | (x << 16)) & 0x0000ffff0000ffffull;
    x = (x | (x << 8)) & 0x00ff00ff00ff00ffull;
    x = (x | (x << 4)) & 0x0f0f0f0f0f0f0f0full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x | (x << 1);
}

IBS_HD uint64_t low_bits_mask(uint64_t n) { return n >= 64 ? ~0ull : ((1ull << n) - 1); }

// Seq word of contig-local word w: random bases, zero past the contig end and
// under N (as the reference's packWindow writes code 0 for a non-ACGT byte).
IBS_HD uint64_t packed_word(uint64_t seed, uint32_t c, uint64_t w, uint64_t len, uint64_t maskWord)
{
    const uint64_t b0 = w * 32;
    if (b0 >= len)
        return 0;
    uint64_t x = base_word(seed, c, w);
    const uint64_t valid = len - b0 >= 32 ? ~0ull : low_bits_mask(2 * (len - b0));
    const uint32_t m = (uint32_t)(maskWord >> (32 * (w & 1)));
    return x & valid & ~spread2(m);
}

SampleParams sample_params(const ibs_synth_sample_spec *s)
{
    SampleParams p{};
    p.seed = s->seed;
    p.k = s->k;
    p.nClasses = std::max(1u, std::min(4u, s->n_classes));
    p.blockLen = s->block_len ? s->block_len : (1ull << 20);
    auto scale = [](double x) -> uint64_t {
        if (x <= 0)
            return 0;
        if (x >= 1)
            return ~0ull;
        return (uint64_t)std::ldexp(x, 64);
    };
    double cum = 0;
    for (uint32_t j = 0; j < 4; ++j) {
        cum += j < p.nClasses ? s->class_prob[j] : 0;
        p.classCut[j] = j + 1 >= p.nClasses ? ~0ull : scale(cum);
        p.classThr[j] = j < p.nClasses ? scale(s->class_rate[j]) : 0;
    }
    p.presentThr = s->present_frac >= 1 ? ~0ull : scale(s->present_frac);
    p.introThr = scale(s->intro_rate);
    return p;
}

// Per-contig list of introgression ranges.
struct Intro {
    uint64_t start, end;
};

// ---------------------------------------------------------------------------
// device kernels
// ---------------------------------------------------------------------------
__global__ void k_mask_runs(const uint32_t *rc, const uint64_t *rs, const uint64_t *rl, uint64_t n,
                            const uint64_t *off, unsigned long long *mask)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b0 = off[rc[i]] + rs[i], b1 = b0 + rl[i];
        for (uint64_t b = b0; b < b1;) {
            const uint64_t w = b >> 6, lo = b & 63;
            const uint64_t hi = std::min<uint64_t>(64, lo + (b1 - b));
            const uint64_t bits = low_bits_mask(hi - lo) << lo;
            atomicOr(mask + w, (unsigned long long)bits);
            b += hi - lo;
        }
    }
}

__global__ void k_seq_words(uint64_t seed, const uint64_t *wordOff, const uint64_t *lens,
                            uint32_t nContigs, uint64_t totalWords, const uint64_t *mask,
                            uint64_t *seq)
{
    for (uint64_t gw = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gw < totalWords;
         gw += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nContigs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (wordOff[mid] <= gw)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint64_t w = gw - wordOff[lo];
        seq[gw] = packed_word(seed, lo, w, lens[lo], mask[gw >> 1]);
    }
}

// The sample copy, packed like the reference.
__global__ void k_copy_words(SampleParams sp, const uint64_t *wordOff, const uint64_t *lens,
                             uint32_t nContigs, uint64_t totalWords, const uint64_t *refSeq,
                             const Intro *intro, const uint32_t *introOff, uint64_t *copy)
{
    for (uint64_t gw = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; gw < totalWords;
         gw += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nContigs - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (wordOff[mid] <= gw)
                lo = mid;
            else
                hi = mid - 1;
        }
        const uint32_t c = lo;
        const uint64_t w = gw - wordOff[c];
        const uint64_t len = lens[c];
        const uint64_t in = refSeq[gw];
        uint64_t out = 0;
        for (uint32_t t = 0; t < 32; ++t) {
            const uint64_t i = w * 32 + t;
            if (i >= len)
                break;
            uint64_t thr = snp_threshold_of_block(sp, c, i / sp.blockLen);
            for (uint32_t j = introOff[c]; j < introOff[c + 1]; ++j)
                if (i >= intro[j].start && i < intro[j].end)
                    thr = sp.introThr;
            const uint32_t b = copy_base(sp, c, i, (uint32_t)(in >> (2 * t)) & 3, thr);
            out |= (uint64_t)b << (2 * t);
        }
        copy[gw] = out;
    }
}

// Canonical k-mers of the copy at valid, present positions; appended through
// a global counter (warp-aggregated).
__global__ void k_sample_kmers(SampleParams sp, const uint64_t *baseOff, const uint64_t *lens,
                               uint32_t nContigs, uint64_t totalBases, const uint64_t *copy,
                               const uint64_t *mask, uint64_t *out, uint64_t cap,
                               unsigned long long *count)
{
    const uint32_t k = sp.k;
    const uint64_t kmask = key_mask(2 * k), kbits = (1ull << k) - 1;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nIter = (totalBases + stride - 1) / stride;
    for (uint64_t it = 0; it < nIter; ++it) {
        const uint64_t G = it * stride + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
        bool emit = false;
        uint64_t code = 0;
        if (G < totalBases) {
            uint32_t lo = 0, hi = nContigs - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (baseOff[mid] <= G)
                    lo = mid;
                else
                    hi = mid - 1;
            }
            const uint64_t i = G - baseOff[lo];
            if (lens[lo] >= k && i <= lens[lo] - k && block_present(sp, lo, i / sp.blockLen)) {
                const uint64_t wi = G >> 5;
                const uint32_t sh = (uint32_t)(G & 31) * 2;
                const uint64_t x = (copy[wi] >> sh) | ((copy[wi + 1] << (63 - sh)) << 1);
                const uint32_t ms = (uint32_t)(G & 63);
                const uint64_t mm = (mask[G >> 6] >> ms) | ((mask[(G >> 6) + 1] << (63 - ms)) << 1);
                if ((mm & kbits) == 0) {
                    uint64_t y = __brevll(x);
                    y = ((y >> 1) & 0x5555555555555555ull) | ((y & 0x5555555555555555ull) << 1);
                    const uint64_t fwd = y >> (64 - 2 * k), rc = ~x & kmask;
                    code = fwd < rc ? fwd : rc;
                    emit = true;
                }
            }
        }
        const uint32_t ballot = __ballot_sync(0xffffffffu, emit);
        if (!ballot)
            continue;
        unsigned long long base = 0;
        if (lane == 0)
            base = atomicAdd(count, (unsigned long long)__popc(ballot));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (emit) {
            const uint64_t idx = base + __popc(ballot & ((1u << lane) - 1u));
            if (idx < cap)
                out[idx] = code;
        }
    }
}

__global__ void k_random_kmers(uint64_t seed, uint32_t k, uint64_t n, uint64_t *out)
{
    const uint64_t kmask = key_mask(2 * k);
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x * blockDim.x)
        out[j] = canonical_of(rnd(seed, S_RAND, j) & kmask, k);
}

__global__ void k_bins(const uint64_t *codes, uint64_t n, uint32_t k, uint32_t sigLen,
                       uint32_t nBins, const uint32_t *norm, uint32_t *bins)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        bins[i] = sigLen ? bin_of_signature(signature_of(codes[i], k, sigLen, norm), nBins) : 0;
}

__global__ void k_lut_hist(const uint64_t *codes, const uint32_t *bins, uint64_t n, uint32_t sufBits,
                           uint64_t single, unsigned long long *hist)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t prefix = sufBits >= 64 ? 0 : codes[i] >> sufBits;
        atomicAdd(hist + (uint64_t)bins[i] * single + prefix, 1ull);
    }
}

__global__ void k_records(const uint64_t *codes, uint64_t r0, uint64_t n, uint32_t sufBytes,
                          uint32_t cntBytes, uint64_t countSeed, uint32_t maxCount, uint8_t *out)
{
    const uint32_t rec = sufBytes + cntBytes;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t code = codes[r0 + i];
        uint8_t *q = out + i * rec;
        for (uint32_t b = 0; b < sufBytes; ++b)
            q[b] = (uint8_t)(code >> (8 * (sufBytes - 1 - b)));
        uint32_t cnt = count_of(countSeed, code);
        cnt = cnt > maxCount ? maxCount : cnt;
        for (uint32_t b = 0; b < cntBytes; ++b)
            q[sufBytes + b] = (uint8_t)(cnt >> (8 * b));
    }
}

int grid_for(uint64_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256, (uint64_t)sms * 16));
}

template <typename T> struct DevBuf {
    T *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    cudaError_t alloc(uint64_t n) { return cudaMalloc(&p, std::max<uint64_t>(n, 1) * sizeof(T)); }
};

// ---------------------------------------------------------------------------
// KMC writer core
// ---------------------------------------------------------------------------
ibs_status check_kmc_spec(const ibs_kmc_spec *s, uint32_t maxK = 32)
{
    if (!s || s->k == 0 || s->k > maxK || s->p > s->k || (s->k - s->p) % 4 != 0 || s->p > 15)
        return fail(IBS_ERR_ARG, "kmc spec: need k <= " + std::to_string(maxK) +
                                     ", p <= 15 and (k - p) % 4 == 0");
    if (s->counter_size > 4)
        return fail(IBS_ERR_ARG, "kmc spec: counter_size must be 0..4");
    if (s->version != 0 && s->version != 0x200)
        return fail(IBS_ERR_ARG, "kmc spec: version must be 0 or 0x200");
    if (s->version == 0x200 && (s->sig_len < 5 || s->sig_len > 11 || s->sig_len > s->k || s->n_bins == 0))
        return fail(IBS_ERR_ARG, "kmc spec: sig_len must be 5..11 and <= k, and n_bins > 0");
    return IBS_OK;
}

uint32_t max_count_of(const ibs_kmc_spec *s)
{
    if (s->counter_size == 0)
        return 1;
    if (s->counter_size >= 4)
        return 0xffffffffu;
    return (1u << (8 * s->counter_size)) - 1;
}

ibs_status write_pre(const std::string &path, const ibs_kmc_spec *s, const std::vector<uint64_t> &lut,
                     uint64_t total)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f)
        return fail(IBS_ERR_IO, "cannot write " + path);
    bool ok = fwrite("KMCP", 1, 4, f) == 4;
    ok = ok && fwrite(lut.data(), 8, lut.size(), f) == lut.size();
    if (s->version == 0x200) {
        const uint32_t nSig = (1u << (2 * s->sig_len)) + 1;
        std::vector<uint32_t> sig(nSig);
        for (uint32_t i = 0; i < nSig; ++i)
            sig[i] = bin_of_signature(i, s->n_bins);
        ok = ok && fwrite(sig.data(), 4, nSig, f) == nSig;
    }
    uint8_t hdr[64];
    memset(hdr, 0, sizeof hdr);
    auto put32 = [&](int at, uint32_t v) { memcpy(hdr + at, &v, 4); };
    const uint32_t minC = s->min_count, maxC = s->max_count ? s->max_count : max_count_of(s);
    put32(0, s->k);
    put32(4, 0); // mode 0: plain counters
    put32(8, s->counter_size);
    put32(12, s->p);
    if (s->version == 0x200) {
        put32(16, s->sig_len);
        put32(20, minC);
        put32(24, maxC);
        memcpy(hdr + 28, &total, 8);
        hdr[36] = 0; // both strands (the reader stores its negation)
    } else {
        put32(16, minC);
        put32(20, maxC);
        memcpy(hdr + 24, &total, 8);
        hdr[32] = 0;
        put32(33, 0); // max_count high word
    }
    put32(60, s->version);
    ok = ok && fwrite(hdr, 1, 64, f) == 64;
    const uint32_t hoff = 64;
    ok = ok && fwrite(&hoff, 4, 1, f) == 1;
    ok = ok && fwrite("KMCP", 1, 4, f) == 4;
    ok = (fclose(f) == 0) && ok;
    return ok ? IBS_OK : fail(IBS_ERR_IO, "short write to " + path);
}

std::vector<uint32_t> norm_table(uint32_t len)
{
    std::vector<uint32_t> n((size_t)1 << (2 * len));
    for (uint32_t i = 0; i < n.size(); ++i)
        n[i] = norm_value(i, len);
    return n;
}

} // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" const char *ibs_tools_last_error(void) { return g_err.c_str(); }

extern "C" uint64_t ibs_synth_n_runs(const ibs_synth_ref_spec *s, uint32_t *contig, uint64_t *start,
                                     uint64_t *len, uint64_t cap)
{
    const auto runs = make_runs(s, S_NRUN, s->n_frac, s->n_run_min, s->n_run_max);
    for (uint64_t i = 0; i < runs.size() && i < cap; ++i) {
        if (contig)
            contig[i] = runs[i].c;
        if (start)
            start[i] = runs[i].start;
        if (len)
            len[i] = runs[i].len;
    }
    return runs.size();
}

extern "C" ibs_status ibs_synth_reference(const ibs_synth_ref_spec *s, uint64_t *seq, uint64_t *mask,
                                          int on_device)
{
    if (!s || (s->n_contigs && !s->lens) || !seq || !mask)
        return fail(IBS_ERR_ARG, "ibs_synth_reference: bad argument");
    std::vector<uint64_t> off;
    uint64_t seqWords, maskWords;
    offsets(s, off, seqWords, maskWords);
    const auto runs = make_runs(s, S_NRUN, s->n_frac, s->n_run_min, s->n_run_max);
    if (!on_device) {
        memset(mask, 0, maskWords * 8);
        for (const Run &r : runs)
            for (uint64_t b = off[r.c] + r.start, e = b + r.len; b < e; ++b)
                mask[b >> 6] |= 1ull << (b & 63);
        std::vector<uint64_t> wordOff(s->n_contigs);
        for (uint32_t c = 0; c < s->n_contigs; ++c)
            wordOff[c] = off[c] / 32;
        seq[seqWords - 1] = 0;
        parallel_for(s->n_contigs, hw_threads(), [&](uint64_t c) {
            const uint64_t nw = round_up64(s->lens[c]) / 32;
            for (uint64_t w = 0; w < nw; ++w) {
                const uint64_t gw = wordOff[c] + w;
                seq[gw] = packed_word(s->seed, (uint32_t)c, w, s->lens[c], mask[gw >> 1]);
            }
        });
        return IBS_OK;
    }
    if (s->n_contigs == 0) {
        TCUDA(cudaMemset(seq, 0, seqWords * 8), "synth");
        TCUDA(cudaMemset(mask, 0, maskWords * 8), "synth");
        return IBS_OK;
    }
    DevBuf<uint32_t> rc;
    DevBuf<uint64_t> rs, rl, dOff, wOff, dLens;
    const uint64_t nr = runs.size();
    std::vector<uint32_t> hc(nr);
    std::vector<uint64_t> hs(nr), hl(nr), wo(s->n_contigs);
    for (uint64_t i = 0; i < nr; ++i)
        hc[i] = runs[i].c, hs[i] = runs[i].start, hl[i] = runs[i].len;
    for (uint32_t c = 0; c < s->n_contigs; ++c)
        wo[c] = off[c] / 32;
    TCUDA(rc.alloc(nr), "synth alloc");
    TCUDA(rs.alloc(nr), "synth alloc");
    TCUDA(rl.alloc(nr), "synth alloc");
    TCUDA(dOff.alloc(s->n_contigs), "synth alloc");
    TCUDA(wOff.alloc(s->n_contigs), "synth alloc");
    TCUDA(dLens.alloc(s->n_contigs), "synth alloc");
    TCUDA(cudaMemcpy(rc.p, hc.data(), nr * 4, cudaMemcpyHostToDevice), "synth upload");
    TCUDA(cudaMemcpy(rs.p, hs.data(), nr * 8, cudaMemcpyHostToDevice), "synth upload");
    TCUDA(cudaMemcpy(rl.p, hl.data(), nr * 8, cudaMemcpyHostToDevice), "synth upload");
    TCUDA(cudaMemcpy(dOff.p, off.data(), s->n_contigs * 8, cudaMemcpyHostToDevice), "synth upload");
    TCUDA(cudaMemcpy(wOff.p, wo.data(), s->n_contigs * 8, cudaMemcpyHostToDevice), "synth upload");
    TCUDA(cudaMemcpy(dLens.p, s->lens, s->n_contigs * 8, cudaMemcpyHostToDevice), "synth upload");
    TCUDA(cudaMemset(mask, 0, maskWords * 8), "synth");
    TCUDA(cudaMemset(seq, 0, seqWords * 8), "synth");
    if (nr)
        k_mask_runs<<<grid_for(nr), 256>>>(rc.p, rs.p, rl.p, nr, dOff.p, (unsigned long long *)mask);
    k_seq_words<<<grid_for(seqWords - 1), 256>>>(s->seed, wOff.p, dLens.p, s->n_contigs,
                                                 seqWords - 1, mask, seq);
    TCUDA(cudaGetLastError(), "synth kernels");
    TCUDA(cudaDeviceSynchronize(), "synth kernels");
    return IBS_OK;
}

extern "C" ibs_status ibs_synth_contig_ascii(const ibs_synth_ref_spec *s, uint32_t c, char *out)
{
    if (!s || c >= s->n_contigs || !out)
        return fail(IBS_ERR_ARG, "ibs_synth_contig_ascii: bad argument");
    const uint64_t len = s->lens[c];
    static const char up[4] = {'A', 'C', 'G', 'T'}, lo[4] = {'a', 'c', 'g', 't'};
    std::vector<uint8_t> flag(len, 0); // bit0 N, bit1 lowercase
    for (const Run &r : make_runs(s, S_NRUN, s->n_frac, s->n_run_min, s->n_run_max))
        if (r.c == c)
            for (uint64_t i = r.start; i < r.start + r.len; ++i)
                flag[i] |= 1;
    for (const Run &r : make_runs(s, S_LOWER, s->lower_frac, s->lower_run_min, s->lower_run_max))
        if (r.c == c)
            for (uint64_t i = r.start; i < r.start + r.len; ++i)
                flag[i] |= 2;
    parallel_for((len + (1 << 22) - 1) >> 22, hw_threads(), [&](uint64_t piece) {
        const uint64_t i0 = piece << 22, i1 = std::min<uint64_t>(len, i0 + (1 << 22));
        for (uint64_t i = i0; i < i1; ++i) {
            if (flag[i] & 1) {
                out[i] = (flag[i] & 2) ? 'n' : 'N';
                continue;
            }
            const uint32_t b = (uint32_t)(base_word(s->seed, c, i / 32) >> (2 * (i % 32))) & 3;
            out[i] = (flag[i] & 2) ? lo[b] : up[b];
        }
    });
    return IBS_OK;
}

extern "C" ibs_status ibs_synth_write_fasta(const ibs_synth_ref_spec *s, const char *path,
                                            const char *const *names, uint32_t width)
{
    if (!s || !path || width == 0)
        return fail(IBS_ERR_ARG, "ibs_synth_write_fasta: bad argument");
    FILE *f = fopen(path, "wb");
    if (!f)
        return fail(IBS_ERR_IO, std::string("cannot write ") + path);
    bool ok = true;
    std::vector<char> buf, text;
    for (uint32_t c = 0; c < s->n_contigs && ok; ++c) {
        const uint64_t len = s->lens[c];
        buf.resize(len);
        ibs_status st = ibs_synth_contig_ascii(s, c, buf.data());
        if (st != IBS_OK) {
            fclose(f);
            return st;
        }
        std::string name = names && names[c] ? names[c] : ("chr" + std::to_string(c + 1));
        ok = fprintf(f, ">%s\n", name.c_str()) > 0;
        text.resize(len + len / width + 2);
        uint64_t o = 0;
        for (uint64_t i = 0; i < len; i += width) {
            const uint64_t m = std::min<uint64_t>(width, len - i);
            memcpy(text.data() + o, buf.data() + i, m);
            o += m;
            text[o++] = '\n';
        }
        ok = ok && fwrite(text.data(), 1, o, f) == o;
    }
    ok = (fclose(f) == 0) && ok;
    return ok ? IBS_OK : fail(IBS_ERR_IO, std::string("short write to ") + path);
}

static std::vector<std::vector<Intro>> intro_lists(const ibs_synth_ref_spec *r,
                                                   const ibs_synth_sample_spec *s)
{
    std::vector<std::vector<Intro>> v(r->n_contigs);
    for (uint32_t j = 0; j < s->n_intro; ++j)
        if (s->intro_contig[j] < r->n_contigs)
            v[s->intro_contig[j]].push_back({s->intro_start[j], s->intro_start[j] + s->intro_len[j]});
    return v;
}

static uint64_t random_count(const ibs_synth_ref_spec *r, const ibs_synth_sample_spec *s)
{
    uint64_t tot = 0;
    for (uint32_t c = 0; c < r->n_contigs; ++c)
        tot += r->lens[c];
    return (uint64_t)((double)tot * s->random_frac);
}

extern "C" ibs_status ibs_synth_sample_codes(const ibs_synth_ref_spec *r, const ibs_synth_sample_spec *s,
                                             const uint64_t *seq, const uint64_t *mask, int on_device,
                                             uint64_t *codes, uint64_t cap, uint64_t *n_out)
{
    if (!r || !s || !n_out || s->k == 0 || s->k > 32 || !seq || !mask)
        return fail(IBS_ERR_ARG, "ibs_synth_sample_codes: bad argument");
    const SampleParams sp = sample_params(s);
    std::vector<uint64_t> off;
    uint64_t seqWords, maskWords;
    offsets(r, off, seqWords, maskWords);
    const uint64_t nRand = random_count(r, s);
    const auto intro = intro_lists(r, s);
    const uint32_t k = s->k;
    if (on_device) {
        uint64_t upper = nRand;
        for (uint32_t c = 0; c < r->n_contigs; ++c)
            upper += r->lens[c] >= k ? r->lens[c] - k + 1 : 0;
        *n_out = upper;
        if (!codes)
            return IBS_OK;
        if (r->n_contigs == 0) {
            k_random_kmers<<<grid_for(nRand), 256>>>(s->seed, k, std::min(nRand, cap), codes);
            TCUDA(cudaDeviceSynchronize(), "synth sample");
            *n_out = std::min(nRand, cap);
            return IBS_OK;
        }
        std::vector<Intro> flat;
        std::vector<uint32_t> introOff(r->n_contigs + 1, 0);
        for (uint32_t c = 0; c < r->n_contigs; ++c) {
            introOff[c] = (uint32_t)flat.size();
            flat.insert(flat.end(), intro[c].begin(), intro[c].end());
        }
        introOff[r->n_contigs] = (uint32_t)flat.size();
        std::vector<uint64_t> wo(r->n_contigs);
        for (uint32_t c = 0; c < r->n_contigs; ++c)
            wo[c] = off[c] / 32;
        DevBuf<uint64_t> copy, dOff, dWo, dLens;
        DevBuf<Intro> dIntro;
        DevBuf<uint32_t> dIntroOff;
        DevBuf<unsigned long long> dCount;
        TCUDA(copy.alloc(seqWords), "synth alloc");
        TCUDA(dOff.alloc(r->n_contigs), "synth alloc");
        TCUDA(dWo.alloc(r->n_contigs), "synth alloc");
        TCUDA(dLens.alloc(r->n_contigs), "synth alloc");
        TCUDA(dIntro.alloc(flat.size()), "synth alloc");
        TCUDA(dIntroOff.alloc(introOff.size()), "synth alloc");
        TCUDA(dCount.alloc(1), "synth alloc");
        TCUDA(cudaMemcpy(dOff.p, off.data(), r->n_contigs * 8, cudaMemcpyHostToDevice), "upload");
        TCUDA(cudaMemcpy(dWo.p, wo.data(), r->n_contigs * 8, cudaMemcpyHostToDevice), "upload");
        TCUDA(cudaMemcpy(dLens.p, r->lens, r->n_contigs * 8, cudaMemcpyHostToDevice), "upload");
        if (!flat.empty())
            TCUDA(cudaMemcpy(dIntro.p, flat.data(), flat.size() * sizeof(Intro), cudaMemcpyHostToDevice),
                  "upload");
        TCUDA(cudaMemcpy(dIntroOff.p, introOff.data(), introOff.size() * 4, cudaMemcpyHostToDevice),
              "upload");
        TCUDA(cudaMemset(dCount.p, 0, 8), "synth");
        TCUDA(cudaMemset(copy.p + seqWords - 1, 0, 8), "synth");
        k_copy_words<<<grid_for(seqWords - 1), 256>>>(sp, dWo.p, dLens.p, r->n_contigs, seqWords - 1,
                                                      seq, dIntro.p, dIntroOff.p, copy.p);
        const uint64_t totalBases = (seqWords - 1) * 32;
        k_sample_kmers<<<grid_for(totalBases), 256>>>(sp, dOff.p, dLens.p, r->n_contigs, totalBases,
                                                      copy.p, mask, codes, cap, dCount.p);
        TCUDA(cudaGetLastError(), "synth sample kernels");
        unsigned long long n = 0;
        TCUDA(cudaMemcpy(&n, dCount.p, 8, cudaMemcpyDeviceToHost), "synth sample");
        const uint64_t nk = std::min<uint64_t>(n, cap);
        const uint64_t nr = cap > nk ? std::min(nRand, cap - nk) : 0;
        if (nr)
            k_random_kmers<<<grid_for(nr), 256>>>(s->seed, k, nr, codes + nk);
        TCUDA(cudaDeviceSynchronize(), "synth sample");
        *n_out = nk + nr;
        return IBS_OK;
    }
    // host: per contig, the copy rolled base by base
    std::vector<uint64_t> start(r->n_contigs + 1, 0);
    for (uint32_t c = 0; c < r->n_contigs; ++c)
        start[c + 1] = start[c] + (r->lens[c] >= k ? r->lens[c] - k + 1 : 0);
    std::vector<uint64_t> got(r->n_contigs, 0);
    std::vector<std::vector<uint64_t>> per(r->n_contigs);
    parallel_for(r->n_contigs, hw_threads(), [&](uint64_t cc) {
        const uint32_t c = (uint32_t)cc;
        const uint64_t len = r->lens[c];
        auto &v = per[c];
        if (len < k)
            return;
        v.reserve(len - k + 1);
        const uint64_t kmask = key_mask(2 * k);
        const uint32_t rcShift = 2 * (k - 1);
        uint64_t fwd = 0, rcv = 0;
        uint32_t validBases = 0;
        for (uint64_t i = 0; i < len; ++i) {
            const uint64_t G = off[c] + i;
            const bool isN = (mask[G >> 6] >> (G & 63)) & 1;
            const uint32_t rb = (uint32_t)(seq[G >> 5] >> (2 * (G & 31))) & 3;
            uint64_t thr = snp_threshold_of_block(sp, c, i / sp.blockLen);
            for (const Intro &in : intro[c])
                if (i >= in.start && i < in.end)
                    thr = sp.introThr;
            const uint32_t b = copy_base(sp, c, i, rb, thr);
            validBases = isN ? 0 : validBases + 1;
            fwd = ((fwd << 2) | b) & kmask;
            rcv = (rcv >> 2) | ((uint64_t)(3 - b) << rcShift);
            if (i + 1 >= k && validBases >= k) {
                const uint64_t p = i + 1 - k;
                if (block_present(sp, c, p / sp.blockLen))
                    v.push_back(fwd < rcv ? fwd : rcv);
            }
        }
    });
    uint64_t n = 0;
    for (auto &v : per)
        n += v.size();
    *n_out = n + nRand;
    if (!codes)
        return IBS_OK;
    uint64_t o = 0;
    for (auto &v : per)
        for (uint64_t x : v)
            if (o < cap)
                codes[o++] = x;
    const uint64_t kmask = key_mask(2 * k);
    for (uint64_t j = 0; j < nRand && o < cap; ++j)
        codes[o++] = canonical_of(rnd(s->seed, S_RAND, j) & kmask, k);
    *n_out = o;
    return IBS_OK;
}

extern "C" uint64_t ibs_sort_unique_host(uint64_t *codes, uint64_t n, int threads)
{
    if (n < 2)
        return n;
    if (threads <= 0)
        threads = hw_threads();
    // parallel: sort pieces, then merge pairwise
    const uint64_t pieces = std::min<uint64_t>((uint64_t)threads, std::max<uint64_t>(1, n >> 20));
    std::vector<uint64_t> cut(pieces + 1);
    for (uint64_t i = 0; i <= pieces; ++i)
        cut[i] = n * i / pieces;
    parallel_for(pieces, threads, [&](uint64_t i) { std::sort(codes + cut[i], codes + cut[i + 1]); });
    for (uint64_t step = 1; step < pieces; step *= 2) {
        std::vector<uint64_t> jobs;
        for (uint64_t i = 0; i + step < pieces; i += 2 * step)
            jobs.push_back(i);
        parallel_for(jobs.size(), threads, [&](uint64_t j) {
            const uint64_t i = jobs[j];
            const uint64_t e = std::min(pieces, i + 2 * step);
            std::inplace_merge(codes + cut[i], codes + cut[i + step], codes + cut[e]);
        });
    }
    return (uint64_t)(std::unique(codes, codes + n) - codes);
}

extern "C" ibs_status ibs_kmc_write(const char *prefix, const ibs_kmc_spec *s, const uint64_t *codes,
                                    uint64_t n, int on_device, uint64_t *n_written)
{
    ibs_status st = check_kmc_spec(s);
    if (st != IBS_OK)
        return st;
    if (!prefix || (n && !codes))
        return fail(IBS_ERR_ARG, "ibs_kmc_write: bad argument");
    const uint32_t k = s->k, p = s->p;
    const uint32_t sufBytes = (k - p) / 4, sufBits = 2 * (k - p);
    const uint32_t rec = sufBytes + s->counter_size;
    const uint64_t single = 1ull << (2 * p);
    const uint32_t nBins = s->version == 0x200 ? s->n_bins : 1;
    const uint32_t sigLen = s->version == 0x200 ? s->sig_len : 0;
    const uint32_t maxCount = max_count_of(s);
    const std::string pre = std::string(prefix) + ".kmc_pre", suf = std::string(prefix) + ".kmc_suf";
    const std::vector<uint32_t> norm = sigLen ? norm_table(sigLen) : std::vector<uint32_t>();
    std::vector<uint64_t> lut((uint64_t)nBins * single + 1, 0);

    if (!on_device) {
        // bin, then per-bin sort + unique
        std::vector<uint32_t> bin(n);
        parallel_for((n + (1 << 20) - 1) >> 20, hw_threads(), [&](uint64_t piece) {
            const uint64_t a = piece << 20, b = std::min<uint64_t>(n, a + (1 << 20));
            for (uint64_t i = a; i < b; ++i)
                bin[i] = sigLen ? bin_of_signature(signature_of(codes[i], k, sigLen, norm.data()), nBins) : 0;
        });
        std::vector<uint64_t> binStart(nBins + 1, 0);
        for (uint64_t i = 0; i < n; ++i)
            binStart[bin[i] + 1]++;
        for (uint32_t b = 0; b < nBins; ++b)
            binStart[b + 1] += binStart[b];
        std::vector<uint64_t> sorted(n), fill(binStart.begin(), binStart.end() - 1);
        for (uint64_t i = 0; i < n; ++i)
            sorted[fill[bin[i]]++] = codes[i];
        std::vector<uint64_t> binLen(nBins);
        parallel_for(nBins, hw_threads(), [&](uint64_t b) {
            uint64_t *a = sorted.data() + binStart[b], *e = sorted.data() + binStart[b + 1];
            std::sort(a, e);
            binLen[b] = (uint64_t)(std::unique(a, e) - a);
        });
        uint64_t total = 0;
        FILE *f = fopen(suf.c_str(), "wb");
        if (!f)
            return fail(IBS_ERR_IO, "cannot write " + suf);
        bool ok = fwrite("KMCS", 1, 4, f) == 4;
        std::vector<uint8_t> buf;
        for (uint32_t b = 0; b < nBins; ++b) {
            const uint64_t *a = sorted.data() + binStart[b];
            const uint64_t m = binLen[b];
            // LUT of this bin: first record of each prefix
            uint64_t j = 0;
            for (uint64_t q = 0; q < single; ++q) {
                lut[(uint64_t)b * single + q] = total + j;
                while (j < m && (sufBits >= 64 ? 0 : (a[j] >> sufBits)) == q)
                    ++j;
            }
            buf.resize(m * rec);
            for (uint64_t i = 0; i < m; ++i) {
                uint8_t *q = buf.data() + i * rec;
                for (uint32_t x = 0; x < sufBytes; ++x)
                    q[x] = (uint8_t)(a[i] >> (8 * (sufBytes - 1 - x)));
                uint32_t cnt = count_of(s->count_seed, a[i]);
                cnt = cnt > maxCount ? maxCount : cnt;
                for (uint32_t x = 0; x < s->counter_size; ++x)
                    q[sufBytes + x] = (uint8_t)(cnt >> (8 * x));
            }
            ok = ok && fwrite(buf.data(), 1, buf.size(), f) == buf.size();
            total += m;
        }
        ok = ok && fwrite("KMCS", 1, 4, f) == 4;
        ok = (fclose(f) == 0) && ok;
        if (!ok)
            return fail(IBS_ERR_IO, "short write to " + suf);
        lut[(uint64_t)nBins * single] = total;
        if (n_written)
            *n_written = total;
        return write_pre(pre, s, lut, total);
    }

    // device path: sort codes, unique, bins, stable sort by bin, LUT, records
    DevBuf<uint64_t> a, b;
    DevBuf<uint32_t> binA, binB, dNorm;
    DevBuf<unsigned long long> hist, nUnique;
    DevBuf<uint8_t> temp;
    size_t tempBytes = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0;
    TCUDA(a.alloc(n), "kmc alloc");
    TCUDA(b.alloc(n), "kmc alloc");
    TCUDA(nUnique.alloc(1), "kmc alloc");
    TCUDA(cub::DeviceRadixSort::SortKeys(nullptr, t1, codes, b.p, n, 0, 2 * k), "kmc sort size");
    TCUDA(cub::DeviceSelect::Unique(nullptr, t2, b.p, a.p, nUnique.p, (int64_t)n), "kmc unique size");
    TCUDA(cub::DeviceRadixSort::SortPairs(nullptr, t3, binA.p, binB.p, a.p, b.p, n, 0, 32), "size");
    TCUDA(cub::DeviceScan::ExclusiveSum(nullptr, t4, hist.p, hist.p, (uint64_t)nBins * single), "size");
    tempBytes = std::max(std::max(t1, t2), std::max(t3, t4));
    TCUDA(temp.alloc(tempBytes), "kmc temp alloc");
    TCUDA(cub::DeviceRadixSort::SortKeys(temp.p, tempBytes, codes, b.p, n, 0, 2 * k), "kmc sort");
    TCUDA(cub::DeviceSelect::Unique(temp.p, tempBytes, b.p, a.p, nUnique.p, (int64_t)n), "kmc unique");
    unsigned long long total = 0;
    TCUDA(cudaMemcpy(&total, nUnique.p, 8, cudaMemcpyDeviceToHost), "kmc unique count");
    TCUDA(binA.alloc(total), "kmc alloc");
    TCUDA(binB.alloc(total), "kmc alloc");
    if (sigLen) {
        TCUDA(dNorm.alloc(norm.size()), "kmc alloc");
        TCUDA(cudaMemcpy(dNorm.p, norm.data(), norm.size() * 4, cudaMemcpyHostToDevice), "kmc norm");
    }
    k_bins<<<grid_for(total), 256>>>(a.p, total, k, sigLen, nBins, dNorm.p, binA.p);
    uint32_t binBits = 1;
    while ((1u << binBits) < nBins)
        ++binBits;
    TCUDA(cub::DeviceRadixSort::SortPairs(temp.p, tempBytes, binA.p, binB.p, a.p, b.p, total, 0,
                                          (int)binBits),
          "kmc bin sort");
    // b = codes in (bin, code) order; binB = their bins
    TCUDA(hist.alloc((uint64_t)nBins * single), "kmc alloc");
    TCUDA(cudaMemset(hist.p, 0, (uint64_t)nBins * single * 8), "kmc hist");
    k_lut_hist<<<grid_for(total), 256>>>(b.p, binB.p, total, sufBits, single, hist.p);
    TCUDA(cub::DeviceScan::ExclusiveSum(temp.p, tempBytes, hist.p, hist.p, (uint64_t)nBins * single),
          "kmc scan");
    TCUDA(cudaMemcpy(lut.data(), hist.p, (uint64_t)nBins * single * 8, cudaMemcpyDeviceToHost), "kmc lut");
    lut[(uint64_t)nBins * single] = total;
    // records in 256 MB pieces
    FILE *f = fopen(suf.c_str(), "wb");
    if (!f)
        return fail(IBS_ERR_IO, "cannot write " + suf);
    bool ok = fwrite("KMCS", 1, 4, f) == 4;
    const uint64_t pieceRecs = std::max<uint64_t>(1, (256ull << 20) / rec);
    DevBuf<uint8_t> dRec;
    uint8_t *hRec = nullptr;
    cudaError_t e = dRec.alloc(pieceRecs * rec);
    if (e == cudaSuccess)
        e = cudaMallocHost(&hRec, pieceRecs * rec);
    for (uint64_t r0 = 0; e == cudaSuccess && ok && r0 < total; r0 += pieceRecs) {
        const uint64_t m = std::min<uint64_t>(pieceRecs, total - r0);
        k_records<<<grid_for(m), 256>>>(b.p, r0, m, sufBytes, s->counter_size, s->count_seed, maxCount,
                                         dRec.p);
        e = cudaMemcpy(hRec, dRec.p, m * rec, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            ok = fwrite(hRec, 1, m * rec, f) == m * rec;
    }
    cudaFreeHost(hRec);
    ok = ok && fwrite("KMCS", 1, 4, f) == 4;
    ok = (fclose(f) == 0) && ok;
    TCUDA(e, "kmc records");
    if (!ok)
        return fail(IBS_ERR_IO, "short write to " + suf);
    if (n_written)
        *n_written = total;
    return write_pre(pre, s, lut, total);
}

// The writer for 33 <= k <= 64 (host only): the same files with 128-bit
// codes. The signature of a k-mer (its KMC2 bin) is the smallest normalised
// sig_len-mer over its bases, first base first, as for k <= 32.
extern "C" ibs_status ibs_kmc_write128(const char *prefix, const ibs_kmc_spec *s, const ibs_code128 *codes,
                                       uint64_t n, uint64_t *n_written)
{
    ibs_status st = check_kmc_spec(s, 64);
    if (st != IBS_OK)
        return st;
    if (!prefix || (n && !codes))
        return fail(IBS_ERR_ARG, "ibs_kmc_write128: bad argument");
    if (s->k <= 32)
        return fail(IBS_ERR_ARG, "ibs_kmc_write128: k <= 32 codes take ibs_kmc_write");
    typedef unsigned __int128 u128;
    const uint32_t k = s->k, p = s->p;
    const uint32_t sufBytes = (k - p) / 4, sufBits = 2 * (k - p);
    const uint32_t rec = sufBytes + s->counter_size;
    const uint64_t single = 1ull << (2 * p);
    const uint32_t nBins = s->version == 0x200 ? s->n_bins : 1;
    const uint32_t sigLen = s->version == 0x200 ? s->sig_len : 0;
    const uint32_t maxCount = max_count_of(s);
    const std::string pre = std::string(prefix) + ".kmc_pre", suf = std::string(prefix) + ".kmc_suf";
    const std::vector<uint32_t> norm = sigLen ? norm_table(sigLen) : std::vector<uint32_t>();
    auto wide = [](const ibs_code128 &c) { return ((u128)c.hi << 64) | c.lo; };
    auto signature = [&](u128 code) {
        const uint32_t mmask = (1u << (2 * sigLen)) - 1;
        uint32_t str = 0, best = 0xffffffffu;
        for (uint32_t i = 0; i < k; ++i) {
            str = ((str << 2) | (uint32_t)((code >> (2 * (k - 1 - i))) & 3)) & mmask;
            if (i + 1 >= sigLen)
                best = std::min(best, norm[str]);
        }
        return best;
    };
    // (bin, code) order, duplicates removed
    std::vector<std::pair<uint32_t, u128>> keys(n);
    parallel_for((n + (1 << 16) - 1) >> 16, hw_threads(), [&](uint64_t piece) {
        const uint64_t a = piece << 16, b = std::min<uint64_t>(n, a + (1 << 16));
        for (uint64_t i = a; i < b; ++i) {
            const u128 c = wide(codes[i]);
            keys[i] = {sigLen ? bin_of_signature(signature(c), nBins) : 0u, c};
        }
    });
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    std::vector<uint64_t> lut((uint64_t)nBins * single + 1, 0);
    for (const auto &kv : keys)
        lut[(uint64_t)kv.first * single + (uint64_t)(kv.second >> sufBits) + 1]++;
    for (uint64_t i = 0; i + 1 < lut.size(); ++i)
        lut[i + 1] += lut[i];
    const uint64_t total = keys.size();
    FILE *f = fopen(suf.c_str(), "wb");
    if (!f)
        return fail(IBS_ERR_IO, "cannot write " + suf);
    bool ok = fwrite("KMCS", 1, 4, f) == 4;
    std::vector<uint8_t> buf(std::max<uint64_t>(total, 1) * rec);
    for (uint64_t i = 0; i < total; ++i) {
        uint8_t *q = buf.data() + i * rec;
        const u128 c = keys[i].second;
        for (uint32_t x = 0; x < sufBytes; ++x)
            q[x] = (uint8_t)(c >> (8 * (sufBytes - 1 - x)));
        uint32_t cnt = count_of(s->count_seed, (uint64_t)c ^ (uint64_t)(c >> 64) * 0x9e3779b97f4a7c15ull);
        cnt = cnt > maxCount ? maxCount : cnt;
        for (uint32_t x = 0; x < s->counter_size; ++x)
            q[sufBytes + x] = (uint8_t)(cnt >> (8 * x));
    }
    ok = ok && fwrite(buf.data(), 1, total * rec, f) == total * rec;
    ok = ok && fwrite("KMCS", 1, 4, f) == 4;
    ok = (fclose(f) == 0) && ok;
    if (!ok)
        return fail(IBS_ERR_IO, "short write to " + suf);
    if (n_written)
        *n_written = total;
    return write_pre(pre, s, lut, total);
}

// ---------------------------------------------------------------------------
// Random 32-byte-sector read ceiling (a GUPS-style probe): every thread issues
// independent loads of one 32-byte sector at uniformly random sector indexes
// of a device buffer; returns sectors read per second.
// ---------------------------------------------------------------------------
namespace {
template <int ILP>
__global__ void k_random_sectors(const uint4 *__restrict__ buf, uint64_t nSectors, int iters,
                                 uint64_t seed, uint32_t *out)
{
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (int it = 0; it < iters; ++it) {
        uint4 v[ILP][2];
#pragma unroll
        for (int j = 0; j < ILP; ++j) {
            const uint64_t h = fmix64(seed ^ (tid * 0x9e3779b97f4a7c15ull) ^ ((uint64_t)(it * ILP + j) << 40));
            const uint4 *p = buf + 2 * mulhi64(h, nSectors);
            v[j][0] = __ldg(p);
            v[j][1] = __ldg(p + 1);
        }
#pragma unroll
        for (int j = 0; j < ILP; ++j)
            acc ^= v[j][0].x ^ v[j][0].w ^ v[j][1].y ^ v[j][1].z;
    }
    if (acc == 0x9e3779b9u)
        out[0] = acc;
}
} // namespace

extern "C" ibs_status ibs_random_sector_rate(uint64_t bytes, double *sectors_per_s)
{
    if (!sectors_per_s || bytes < (1u << 20))
        return fail(IBS_ERR_ARG, "ibs_random_sector_rate: bad argument");
    DevBuf<uint4> buf;
    DevBuf<uint32_t> out;
    TCUDA(buf.alloc(bytes / 16), "gups alloc");
    TCUDA(out.alloc(1), "gups alloc");
    TCUDA(cudaMemset(buf.p, 0x5a, bytes), "gups init");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t nSectors = bytes / 32;
    const int grid = sms * 8, threads = 256, iters = 128;
    cudaEvent_t a, b;
    TCUDA(cudaEventCreate(&a), "event");
    TCUDA(cudaEventCreate(&b), "event");
    k_random_sectors<4><<<grid, threads>>>(buf.p, nSectors, iters, 1, out.p);
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a);
        k_random_sectors<4><<<grid, threads>>>(buf.p, nSectors, iters, 100 + r, out.p);
        cudaEventRecord(b);
        TCUDA(cudaEventSynchronize(b), "gups");
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    TCUDA(cudaGetLastError(), "gups");
    *sectors_per_s = (double)grid * threads * iters * 4 / (best * 1e-3);
    return IBS_OK;
}
