/*
 * CPU oracle for the fastibs window scan -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the reference GPU-IBS CPU scan path. It exists to
 * check the product (the CUDA library) and to time a CPU baseline; nothing
 * in the product links it. Each function names the reference file:line it
 * follows (paths relative to the reference project root).
 */
#define _GNU_SOURCE
#include "ibs_oracle.h"

#include <errno.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <zlib.h>

static __thread char g_err[512];

static void set_err(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

const char *orc_error(void) { return g_err; }

/* ======================================================================
 * FASTA / FASTQ reader: src/Utils.hpp:170-255 (readSequenceFile) and
 * :127-166 (decompressGzip).
 * ==================================================================== */
struct orc_seqfile {
    size_t n, cap;
    char **ids;
    char **seqs;
    size_t *lens;
};

typedef struct {
    char *p;
    size_t n, cap;
} buf_t;

static int buf_append(buf_t *b, const char *src, size_t n)
{
    if (b->n + n + 1 > b->cap) {
        size_t c = b->cap ? b->cap : 4096;
        while (c < b->n + n + 1)
            c *= 2;
        char *q = (char *)realloc(b->p, c);
        if (!q)
            return -1;
        b->p = q;
        b->cap = c;
    }
    memcpy(b->p + b->n, src, n);
    b->n += n;
    b->p[b->n] = 0;
    return 0;
}

/* decompressGzip (src/Utils.hpp:127-166): the gzip error state is checked
 * after every gzread, so a truncated stream is an error. */
static int read_gzip(const char *path, buf_t *out)
{
    gzFile f = gzopen(path, "rb");
    if (!f) {
        set_err("Failed to open gzip file %s", path);
        return -1;
    }
    gzbuffer(f, 1 << 20);
    char *chunk = (char *)malloc(1 << 20);
    for (;;) {
        int got = gzread(f, chunk, 1 << 20);
        int errnum = Z_OK;
        const char *why = gzerror(f, &errnum);
        if (got < 0 || (errnum != Z_OK && errnum != Z_STREAM_END)) {
            set_err("Failed to decompress %s: %s", path,
                    errnum == Z_BUF_ERROR ? "truncated gzip stream" : (why ? why : "read error"));
            free(chunk);
            gzclose(f);
            return -1;
        }
        if (got == 0)
            break;
        if (buf_append(out, chunk, (size_t)got)) {
            set_err("out of memory");
            free(chunk);
            gzclose(f);
            return -1;
        }
    }
    free(chunk);
    gzclose(f);
    return 0;
}

static int read_plain(const char *path, buf_t *out)
{
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_err("Failed to open file %s", path);
        return -1;
    }
    fseeko(f, 0, SEEK_END);
    off_t sz = ftello(f);
    fseeko(f, 0, SEEK_SET);
    out->p = (char *)malloc((size_t)sz + 1);
    out->cap = (size_t)sz + 1;
    out->n = fread(out->p, 1, (size_t)sz, f);
    out->p[out->n] = 0;
    fclose(f);
    return 0;
}

static int sf_push(orc_seqfile *r, char *id, char *seq, size_t len)
{
    if (r->n == r->cap) {
        size_t c = r->cap ? 2 * r->cap : 16;
        r->ids = (char **)realloc(r->ids, c * sizeof(char *));
        r->seqs = (char **)realloc(r->seqs, c * sizeof(char *));
        r->lens = (size_t *)realloc(r->lens, c * sizeof(size_t));
        r->cap = c;
    }
    r->ids[r->n] = id;
    r->seqs[r->n] = seq;
    r->lens[r->n] = len;
    r->n++;
    return 0;
}

orc_seqfile *orc_read_sequence_file(const char *path, int compressed)
{
    buf_t data = {0};
    if (compressed ? read_gzip(path, &data) : read_plain(path, &data))
        return NULL;
    if (data.n == 0) {
        set_err("Empty file");
        free(data.p);
        return NULL;
    }
    int fastq;
    if (data.p[0] == '>')
        fastq = 0;
    else if (data.p[0] == '@')
        fastq = 1;
    else {
        set_err("Unknown file type");
        free(data.p);
        return NULL;
    }
    const char idChar = fastq ? '@' : '>';
    orc_seqfile *r = (orc_seqfile *)calloc(1, sizeof *r);
    buf_t id = {0}, seq = {0};
    buf_append(&id, "", 0);
    int isQuality = 0;
    size_t pos = 0;
    /* Lines split on '\n' only; the final partial line counts
     * (src/Utils.hpp:201-246). */
    while (pos < data.n) {
        const char *nl = (const char *)memchr(data.p + pos, '\n', data.n - pos);
        size_t eol = nl ? (size_t)(nl - data.p) : data.n;
        const char *line = data.p + pos;
        size_t lineLen = eol - pos;
        pos = eol + 1;
        if (lineLen == 0)
            continue;
        /* A '+' line in FASTQ marks the next line as quality; checked
         * before the quality-line skip, as at src/Utils.hpp:221-231. */
        if (fastq && line[0] == '+') {
            isQuality = 1;
            continue;
        }
        if (isQuality) {
            isQuality = 0;
            continue;
        }
        if (line[0] == idChar) {
            if (seq.n) {
                sf_push(r, id.p, seq.p, seq.n);
                id = (buf_t){0};
                seq = (buf_t){0};
            }
            id.n = 0;
            buf_append(&id, line + 1, lineLen - 1);
        } else {
            buf_append(&seq, line, lineLen);
        }
    }
    if (seq.n)
        sf_push(r, id.p, seq.p, seq.n);
    else {
        free(id.p);
        free(seq.p);
    }
    free(data.p);
    return r;
}

size_t orc_seqfile_count(const orc_seqfile *f) { return f->n; }
const char *orc_seqfile_id(const orc_seqfile *f, size_t i) { return f->ids[i]; }
const char *orc_seqfile_seq(const orc_seqfile *f, size_t i, size_t *len)
{
    if (len)
        *len = f->lens[i];
    return f->seqs[i];
}
void orc_seqfile_free(orc_seqfile *f)
{
    if (!f)
        return;
    for (size_t i = 0; i < f->n; i++) {
        free(f->ids[i]);
        free(f->seqs[i]);
    }
    free(f->ids);
    free(f->seqs);
    free(f->lens);
    free(f);
}

/* ======================================================================
 * KMC random-access index: src/gpu/KmcRaIndex.hpp (readHeaderOf :497-538,
 * loadPre :540-594, loadSuf :596-708, mmerAllowed/buildNorm :712-750) and
 * the probe of src/gpu/ProbeCore.hpp:58-129.
 * ==================================================================== */
typedef unsigned __int128 u128;

struct orc_index {
    uint32_t k, p, sigLen, suffixBytes, counterBytes;
    uint64_t suffixMask, total, singleLutSize;
    uint64_t *lut;
    size_t lutEntries;
    uint32_t *sigMap;
    size_t sigMapEntries;
    uint32_t *norm;
    uint32_t *suf32;
    uint64_t *suf64;
    u128 *suf128;     /* k > 32: suffixes of up to 16 bytes */
    u128 suffixMask128;
};

static int read_at(FILE *f, long long off, void *dst, size_t n, const char *what)
{
    fseeko(f, off, SEEK_SET);
    if (fread(dst, 1, n, f) != n) {
        set_err("KmcRaIndex: short read of %s", what);
        return -1;
    }
    return 0;
}

static uint64_t file_size(FILE *f)
{
    fseeko(f, 0, SEEK_END);
    return (uint64_t)ftello(f);
}

static int check_markers(FILE *f, uint64_t size, const char *marker, const char *path)
{
    char head[4], tail[4];
    if (size < 8 || read_at(f, 0, head, 4, "marker") || read_at(f, (long long)size - 4, tail, 4, "marker"))
        return -1;
    if (memcmp(head, marker, 4) || memcmp(tail, marker, 4)) {
        set_err("KmcRaIndex: bad marker in %s", path);
        return -1;
    }
    return 0;
}

/* mmerAllowed (src/gpu/KmcRaIndex.hpp:714-732), itself CMmer::is_allowed. */
static int mmer_allowed(uint32_t mmer, uint32_t len)
{
    if ((mmer & 0x3f) == 0x3f)
        return 0;
    if ((mmer & 0x3f) == 0x3b)
        return 0;
    if ((mmer & 0x3c) == 0x3c)
        return 0;
    for (uint32_t j = 0; j < len - 3; ++j) {
        if ((mmer & 0xf) == 0)
            return 0;
        mmer >>= 2;
    }
    if (mmer == 0)
        return 0;
    if (mmer == 0x04)
        return 0;
    if ((mmer & 0xf) == 0)
        return 0;
    return 1;
}

/* buildNorm (src/gpu/KmcRaIndex.hpp:734-750). */
static uint32_t *build_norm(uint32_t len)
{
    const uint32_t special = 1u << (2 * len);
    uint32_t *norm = (uint32_t *)malloc((size_t)special * 4);
    for (uint32_t i = 0; i < special; ++i) {
        uint32_t rev = 0, m = i;
        for (uint32_t j = 0; j < len; ++j) {
            rev = (rev << 2) | (3 - (m & 3));
            m >>= 2;
        }
        const uint32_t a = mmer_allowed(i, len) ? i : special;
        const uint32_t b = mmer_allowed(rev, len) ? rev : special;
        norm[i] = a < b ? a : b;
    }
    return norm;
}

orc_index *orc_index_open(const char *prefix)
{
    char path[4096];
    snprintf(path, sizeof path, "%s.kmc_pre", prefix);
    FILE *f = fopen(path, "rb");
    if (!f) {
        set_err("KmcRaIndex: cannot open %s", path);
        return NULL;
    }
    orc_index *ix = (orc_index *)calloc(1, sizeof *ix);
    const uint64_t fsize = file_size(f);
    uint32_t version = 0, mode = 0, counterSize = 0;
    unsigned char hoff = 0;
    if (check_markers(f, fsize, "KMCP", path) || read_at(f, (long long)fsize - 12, &version, 4, "version"))
        goto fail;
    if (version != 0 && version != 0x200) {
        set_err("KmcRaIndex: unsupported KMC format version");
        goto fail;
    }
    /* header_offset: only its first byte is read (src/gpu/KmcRaIndex.hpp:511-515). */
    if (read_at(f, (long long)fsize - 8, &hoff, 1, "header offset"))
        goto fail;
    const long long headerPos = (long long)fsize - ((long long)hoff + 8);
    if (version == 0x200) {
        uint32_t h[5];
        if (read_at(f, headerPos, h, sizeof h, "header") ||
            read_at(f, headerPos + 28, &ix->total, 8, "total_kmers"))
            goto fail;
        ix->k = h[0];
        mode = h[1];
        counterSize = h[2];
        ix->p = h[3];
        ix->sigLen = h[4];
    } else {
        uint32_t h[4];
        if (read_at(f, headerPos, h, sizeof h, "header") ||
            read_at(f, headerPos + 24, &ix->total, 8, "total_kmers"))
            goto fail;
        ix->k = h[0];
        mode = h[1];
        counterSize = h[2];
        ix->p = h[3];
        ix->sigLen = 0;
    }
    /* loadPre checks (src/gpu/KmcRaIndex.hpp:551-557). */
    if (mode != 0) {
        set_err("KmcRaIndex: Quake-compatible counters are not supported");
        goto fail;
    }
    /* k > 32: the reference's string path reads the same files through the
     * KMC API (CKMCFile::OpenForRA, KMC/kmc_api/kmc_file.cpp), whose
     * membership test is the same prefix-LUT bucket plus binary search over
     * suffixes (CKMCFile::CheckKmer); suffixes are then up to 16 bytes. */
    if (ix->k == 0 || ix->k > 64) {
        set_err("KmcRaIndex: k=%u is not supported (k must be 1..64)", ix->k);
        goto fail;
    }
    if ((ix->k - ix->p) % 4 != 0 || ix->k - ix->p > (ix->k > 32 ? 64u : 32u)) {
        set_err("KmcRaIndex: unexpected suffix geometry");
        goto fail;
    }
    ix->suffixBytes = (ix->k - ix->p) / 4;
    ix->counterBytes = counterSize;
    {
        const uint32_t sym = ix->k - ix->p;
        ix->suffixMask = sym >= 32 ? ~0ull : (1ull << (2 * sym)) - 1;
        ix->suffixMask128 = sym >= 64 ? ~(u128)0 : (((u128)1 << (2 * sym)) - 1);
    }
    ix->singleLutSize = 1ull << (2 * ix->p);
    if (version == 0x200) {
        ix->sigMapEntries = ((size_t)1 << (2 * ix->sigLen)) + 1;
        const uint64_t sizeNoMarkers = fsize - 12;
        const uint64_t lutAreaBytes = sizeNoMarkers - (ix->sigMapEntries * 4 + hoff + 8);
        ix->lutEntries = (size_t)((lutAreaBytes + 8) / 8);
        ix->lut = (uint64_t *)malloc(ix->lutEntries * 8);
        if (read_at(f, 4, ix->lut, lutAreaBytes + 8, "prefix LUT"))
            goto fail;
        ix->lut[ix->lutEntries - 1] = ix->total + 1; /* KMC's guard quirk */
        ix->sigMap = (uint32_t *)malloc(ix->sigMapEntries * 4);
        if (read_at(f, 4 + (long long)lutAreaBytes + 8, ix->sigMap, ix->sigMapEntries * 4, "signature map"))
            goto fail;
    } else {
        ix->lutEntries = (size_t)ix->singleLutSize + 1;
        ix->lut = (uint64_t *)malloc(ix->lutEntries * 8);
        if (read_at(f, 4, ix->lut, ix->lutEntries * 8, "prefix LUT"))
            goto fail;
        ix->lut[ix->lutEntries - 1] = ix->total + 1;
    }
    fclose(f);
    f = NULL;

    /* loadSuf (src/gpu/KmcRaIndex.hpp:596-708): strip counters, suffix
     * bytes big-endian -> native integer. */
    snprintf(path, sizeof path, "%s.kmc_suf", prefix);
    f = fopen(path, "rb");
    if (!f) {
        set_err("KmcRaIndex: cannot open %s", path);
        goto fail;
    }
    {
        const uint64_t ssize = file_size(f);
        if (check_markers(f, ssize, "KMCS", path))
            goto fail;
        const uint32_t rec = ix->suffixBytes + ix->counterBytes;
        if (ssize - 8 < ix->total * (uint64_t)rec) {
            set_err("KmcRaIndex: suffix file smaller than expected");
            goto fail;
        }
        const int use32 = ix->suffixBytes <= 4, use128 = ix->k > 32;
        if (use128)
            ix->suf128 = (u128 *)malloc(ix->total * 16 + 16);
        else if (use32)
            ix->suf32 = (uint32_t *)malloc(ix->total * 4 + 4);
        else
            ix->suf64 = (uint64_t *)malloc(ix->total * 8 + 8);
        fseeko(f, 4, SEEK_SET);
        const size_t chunkRecs = (1u << 20) / (rec ? rec : 1) + 1;
        unsigned char *buf = (unsigned char *)malloc(chunkRecs * rec + 1);
        uint64_t r = 0;
        while (r < ix->total) {
            size_t batch = (size_t)((ix->total - r) < chunkRecs ? (ix->total - r) : chunkRecs);
            if (fread(buf, 1, batch * rec, f) != batch * rec) {
                set_err("KmcRaIndex: short read of suffix records");
                free(buf);
                goto fail;
            }
            const unsigned char *q = buf;
            for (size_t i = 0; i < batch; i++, q += rec) {
                if (use128) {
                    u128 w = 0;
                    for (uint32_t b = 0; b < ix->suffixBytes; b++)
                        w = (w << 8) | q[b];
                    ix->suf128[r + i] = w;
                    continue;
                }
                uint64_t v = 0;
                for (uint32_t b = 0; b < ix->suffixBytes; b++)
                    v = (v << 8) | q[b];
                if (use32)
                    ix->suf32[r + i] = (uint32_t)v;
                else
                    ix->suf64[r + i] = v;
            }
            r += batch;
        }
        free(buf);
    }
    fclose(f);
    if (ix->sigLen)
        ix->norm = build_norm(ix->sigLen);
    return ix;
fail:
    if (f)
        fclose(f);
    orc_index_close(ix);
    return NULL;
}

void orc_index_close(orc_index *ix)
{
    if (!ix)
        return;
    free(ix->lut);
    free(ix->sigMap);
    free(ix->norm);
    free(ix->suf32);
    free(ix->suf64);
    free(ix->suf128);
    free(ix);
}

void orc_index_params(const orc_index *ix, uint32_t out[6], uint64_t *total)
{
    out[0] = ix->k;
    out[1] = ix->p;
    out[2] = ix->sigLen;
    out[3] = ix->suffixBytes;
    out[4] = ix->counterBytes;
    out[5] = (uint32_t)((ix->lutEntries - 1) / ix->singleLutSize);
    if (total)
        *total = ix->total;
}

/* signatureOf (src/gpu/ProbeCore.hpp:58-76): the minimum norm over the
 * k - sigLen + 1 m-mers of the code, most significant symbol first. */
uint32_t orc_signature(const orc_index *ix, uint64_t code)
{
    const uint32_t k = ix->k, s = ix->sigLen;
    const uint32_t mmask = (1u << (2 * s)) - 1;
    uint32_t str = 0, best = 0xffffffffu;
    for (uint32_t i = 0; i < k; ++i) {
        const uint32_t symb = (uint32_t)(code >> (2 * (k - 1 - i))) & 3;
        str = ((str << 2) | symb) & mmask;
        if (i >= s - 1) {
            const uint32_t v = ix->norm[str];
            if (v < best)
                best = v;
        }
    }
    return best;
}

/* probeOne + probeBucket (src/gpu/ProbeCore.hpp:82-129) over the whole
 * index: prefix range [0, 0xffffffff). */
int orc_probe(const orc_index *ix, uint64_t code)
{
    if (ix->suf128) /* k > 32 indexes answer orc_probe128 only */
        return 0;
    const uint64_t prefix = code >> (2 * (ix->k - ix->p));
    if (prefix >= 0xffffffffu)
        return 0;
    uint64_t lutBase = 0;
    if (ix->sigLen)
        lutBase = (uint64_t)ix->sigMap[orc_signature(ix, code)] * ix->singleLutSize;
    const uint64_t entry = lutBase + prefix;
    long long lo = (long long)ix->lut[entry];
    long long hi = (long long)ix->lut[entry + 1] - 1;
    if (lo >= (long long)ix->total)
        return 0;
    if (hi > (long long)ix->total - 1)
        hi = (long long)ix->total - 1;
    const uint64_t target = code & ix->suffixMask;
    while (lo <= hi) {
        const long long mid = (lo + hi) >> 1;
        const uint64_t s = ix->suf32 ? ix->suf32[mid] : ix->suf64[mid];
        if (s == target)
            return 1;
        if (s < target)
            lo = mid + 1;
        else
            hi = mid - 1;
    }
    return 0;
}

void orc_probe_many(const orc_index *ix, const uint64_t *codes, size_t n, uint8_t *hits)
{
    for (size_t i = 0; i < n; i++)
        hits[i] = (uint8_t)orc_probe(ix, codes[i]);
}

/* forEachKmer / walkBuckets (src/gpu/KmcRaIndex.hpp:169-173, :446-460). */
size_t orc_index_list(const orc_index *ix, uint64_t *codes, size_t cap)
{
    if (ix->suf128) /* k > 32 indexes list through orc_index_list128 */
        return 0;
    const uint32_t shift = 2 * (ix->k - ix->p);
    const uint64_t prefixMask = ix->singleLutSize - 1;
    size_t n = 0;
    for (size_t j = 0; j + 1 < ix->lutEntries; ++j) {
        const uint64_t prefix = ((uint64_t)j & prefixMask) << shift;
        uint64_t lo = ix->lut[j], hi = ix->lut[j + 1];
        if (hi > ix->total)
            hi = ix->total;
        for (uint64_t r = lo; r < hi; ++r) {
            if (n < cap)
                codes[n] = prefix | (ix->suf32 ? (uint64_t)ix->suf32[r] : ix->suf64[r]);
            n++;
        }
    }
    return n;
}

/* The same three for k > 32 (128-bit codes, first base most significant):
 * the signature over the code's m-mers, then the LUT bucket and the binary
 * search, as CKMCFile::CheckKmer does for the string path's
 * CKMCFile::IsKmer (src/KmerDatabase.hpp:689-693). */
static uint32_t signature128(const orc_index *ix, u128 code)
{
    const uint32_t k = ix->k, s = ix->sigLen;
    const uint32_t mmask = (1u << (2 * s)) - 1;
    uint32_t str = 0, best = 0xffffffffu;
    for (uint32_t i = 0; i < k; ++i) {
        const uint32_t symb = (uint32_t)(code >> (2 * (k - 1 - i))) & 3;
        str = ((str << 2) | symb) & mmask;
        if (i >= s - 1) {
            const uint32_t v = ix->norm[str];
            if (v < best)
                best = v;
        }
    }
    return best;
}

int orc_probe128(const orc_index *ix, uint64_t lo, uint64_t hi)
{
    if (!ix->suf128)
        return 0;
    const u128 code = ((u128)hi << 64) | lo;
    const uint64_t prefix = (uint64_t)(code >> (2 * (ix->k - ix->p)));
    uint64_t lutBase = 0;
    if (ix->sigLen)
        lutBase = (uint64_t)ix->sigMap[signature128(ix, code)] * ix->singleLutSize;
    const uint64_t entry = lutBase + prefix;
    long long a = (long long)ix->lut[entry];
    long long b = (long long)ix->lut[entry + 1] - 1;
    if (a >= (long long)ix->total)
        return 0;
    if (b > (long long)ix->total - 1)
        b = (long long)ix->total - 1;
    const u128 target = code & ix->suffixMask128;
    while (a <= b) {
        const long long mid = (a + b) >> 1;
        const u128 v = ix->suf128[mid];
        if (v == target)
            return 1;
        if (v < target)
            a = mid + 1;
        else
            b = mid - 1;
    }
    return 0;
}

size_t orc_index_list128(const orc_index *ix, uint64_t *lo, uint64_t *hi, size_t cap)
{
    if (!ix->suf128)
        return 0;
    const uint32_t shift = 2 * (ix->k - ix->p);
    const uint64_t prefixMask = ix->singleLutSize - 1;
    size_t n = 0;
    for (size_t j = 0; j + 1 < ix->lutEntries; ++j) {
        const u128 prefix = (u128)((uint64_t)j & prefixMask) << shift;
        uint64_t a = ix->lut[j], b = ix->lut[j + 1];
        if (b > ix->total)
            b = ix->total;
        for (uint64_t r = a; r < b; ++r) {
            if (n < cap) {
                const u128 c = prefix | ix->suf128[r];
                lo[n] = (uint64_t)c;
                hi[n] = (uint64_t)(c >> 64);
            }
            n++;
        }
    }
    return n;
}

/* ======================================================================
 * Codec: KmerCodec::getCanonicalCodes (src/KmerCodec.hpp:38-61) with the
 * table of :105-118 (ACGT and acgt valid, every other byte invalid).
 * ==================================================================== */
static unsigned char g_tab[256];
static pthread_once_t g_tab_once = PTHREAD_ONCE_INIT;
static void init_tab(void)
{
    memset(g_tab, 4, sizeof g_tab);
    g_tab['A'] = g_tab['a'] = 0;
    g_tab['C'] = g_tab['c'] = 1;
    g_tab['G'] = g_tab['g'] = 2;
    g_tab['T'] = g_tab['t'] = 3;
}

size_t orc_canonical_codes(const char *seq, size_t len, uint32_t k, uint64_t *codes)
{
    pthread_once(&g_tab_once, init_tab);
    size_t n = 0;
    if (len < k)
        return 0;
    const uint64_t mask = k == 32 ? ~0ull : (1ull << (2 * k)) - 1;
    const uint32_t rcShift = 2 * (k - 1);
    uint64_t fwd = 0, rc = 0;
    uint32_t validBases = 0;
    for (size_t j = 0; j < len; ++j) {
        unsigned c = g_tab[(unsigned char)seq[j]];
        if (c > 3) {
            validBases = 0;
            c = 0;
        } else
            ++validBases;
        fwd = ((fwd << 2) | c) & mask;
        rc = (rc >> 2) | ((uint64_t)(3 - c) << rcShift);
        if (validBases >= k)
            codes[n++] = fwd < rc ? fwd : rc;
    }
    return n;
}

/* The string path's k-mers for k > 32: getCanonicalKmersLegacy
 * (src/Utils.hpp:102-125) upper-cases the window, skips every k-mer with a
 * byte outside ACGT and keeps the smaller of the k-mer and its reverse
 * complement as strings; as 2k-bit codes (A<C<G<T) the string order is the
 * integer order. */
size_t orc_canonical_codes128(const char *seq, size_t len, uint32_t k, uint64_t *lo, uint64_t *hi)
{
    pthread_once(&g_tab_once, init_tab);
    size_t n = 0;
    if (len < k || k > 64)
        return 0;
    const u128 mask = k == 64 ? ~(u128)0 : (((u128)1 << (2 * k)) - 1);
    const uint32_t rcShift = 2 * (k - 1);
    u128 fwd = 0, rc = 0;
    uint32_t validBases = 0;
    for (size_t j = 0; j < len; ++j) {
        unsigned c = g_tab[(unsigned char)seq[j]];
        if (c > 3) {
            validBases = 0;
            c = 0;
        } else
            ++validBases;
        fwd = ((fwd << 2) | c) & mask;
        rc = (rc >> 2) | ((u128)(3 - c) << rcShift);
        if (validBases >= k) {
            const u128 m = fwd < rc ? fwd : rc;
            lo[n] = (uint64_t)m;
            hi[n] = (uint64_t)(m >> 64);
            n++;
        }
    }
    return n;
}

/* ======================================================================
 * Windows: chunkSequences (src/Utils.hpp:296-327): [j, min(j+W, len)) for
 * j = 0, W-k, 2(W-k), ... while j < len.
 * ==================================================================== */
size_t orc_window_count(size_t len, uint32_t W, uint32_t k)
{
    if (W <= k)
        return 0;
    const size_t step = W - k;
    return len ? (len + step - 1) / step : 0;
}

/* Window::addVariationOriginal (src/Window.hpp:29-36). */
static void add_variation(orc_window *w, int gap, int k)
{
    w->variations += 1;
    int d = gap - (k - 1);
    if (d <= 0)
        d = abs(d + 1);
    w->kmer_distance += d;
}

/* The statistics loop of getStatsFromSequence (src/KmerDatabase.hpp:628-646
 * for CPU-BATCHED, :650-672 for CPU-OPT). */
void orc_stats_from_hits(const uint8_t *hits, size_t n, uint32_t k, orc_window *row)
{
    row->total_kmers = (int32_t)n;
    int gap = 0;
    for (size_t i = 0; i < n; i++) {
        if (!hits[i])
            gap += 1;
        else {
            row->observed_kmers += 1;
            if (gap > 0) {
                add_variation(row, gap, (int)k);
                gap = 0;
            }
        }
    }
    if (gap > 0)
        add_variation(row, gap, (int)k);
}

static int pred_hit(uint64_t code) { return (code * 0x9E3779B97F4A7C15ull >> 61) == 0; }

/* codes holds 2 (W + 1) words: the low words, then (k > 32) the high words. */
static void scan_window(const orc_index *ix, const char *seq, size_t len, size_t j, uint32_t W,
                        uint32_t k, orc_window *row, uint64_t *codes, uint8_t *hits)
{
    const size_t end = j + W > len ? len : j + W;
    memset(row, 0, sizeof *row);
    row->start = (int32_t)j;
    row->end = (int32_t)end;
    if (k > 32) {
        uint64_t *hi = codes + W + 1;
        const size_t n = orc_canonical_codes128(seq + j, end - j, k, codes, hi);
        for (size_t i = 0; i < n; i++)
            hits[i] = (uint8_t)(ix ? orc_probe128(ix, codes[i], hi[i])
                                   : pred_hit(codes[i] ^ (hi[i] * 0xC2B2AE3D27D4EB4Full)));
        orc_stats_from_hits(hits, n, k, row);
        return;
    }
    const size_t n = orc_canonical_codes(seq + j, end - j, k, codes);
    for (size_t i = 0; i < n; i++)
        hits[i] = (uint8_t)(ix ? orc_probe(ix, codes[i]) : pred_hit(codes[i]));
    orc_stats_from_hits(hits, n, k, row);
}

int orc_scan_contig(const orc_index *ix, const char *seq, size_t len, uint32_t W, uint32_t k,
                    orc_window *rows)
{
    if (W <= k) {
        set_err("window size %u must be larger than k (%u)", W, k);
        return -1;
    }
    uint64_t *codes = (uint64_t *)malloc(((size_t)W + 1) * 16);
    uint8_t *hits = (uint8_t *)malloc((size_t)W + 1);
    size_t w = 0;
    for (size_t j = 0; j < len; j += W - k)
        scan_window(ix, seq, len, j, W, k, &rows[w++], codes, hits);
    free(codes);
    free(hits);
    return 0;
}

typedef struct {
    const orc_index *ix;
    const char *const *seqs;
    const size_t *lens;
    size_t n;
    uint32_t W, k;
    orc_window *rows;
    size_t *rowOff;
    size_t *winContig; /* flat window -> contig */
    size_t nWin;
    size_t next;
    pthread_mutex_t mu;
} scan_job;

static void *scan_worker(void *arg)
{
    scan_job *J = (scan_job *)arg;
    uint64_t *codes = (uint64_t *)malloc(((size_t)J->W + 1) * 16);
    uint8_t *hits = (uint8_t *)malloc((size_t)J->W + 1);
    for (;;) {
        pthread_mutex_lock(&J->mu);
        size_t w0 = J->next;
        J->next += 64;
        pthread_mutex_unlock(&J->mu);
        if (w0 >= J->nWin)
            break;
        size_t w1 = w0 + 64 < J->nWin ? w0 + 64 : J->nWin;
        for (size_t w = w0; w < w1; w++) {
            const size_t c = J->winContig[w];
            const size_t j = (w - J->rowOff[c]) * (J->W - J->k);
            scan_window(J->ix, J->seqs[c], J->lens[c], j, J->W, J->k, &J->rows[w], codes, hits);
        }
    }
    free(codes);
    free(hits);
    return NULL;
}

int orc_scan_contigs(const orc_index *ix, const char *const *seqs, const size_t *lens, size_t n,
                     uint32_t W, uint32_t k, int threads, orc_window *rows)
{
    if (W <= k) {
        set_err("window size %u must be larger than k (%u)", W, k);
        return -1;
    }
    scan_job J;
    memset(&J, 0, sizeof J);
    J.ix = ix;
    J.seqs = seqs;
    J.lens = lens;
    J.n = n;
    J.W = W;
    J.k = k;
    J.rows = rows;
    J.rowOff = (size_t *)malloc((n + 1) * sizeof(size_t));
    size_t tot = 0;
    for (size_t c = 0; c < n; c++) {
        J.rowOff[c] = tot;
        tot += orc_window_count(lens[c], W, k);
    }
    J.rowOff[n] = tot;
    J.nWin = tot;
    J.winContig = (size_t *)malloc((tot + 1) * sizeof(size_t));
    for (size_t c = 0; c < n; c++)
        for (size_t w = J.rowOff[c]; w < J.rowOff[c + 1]; w++)
            J.winContig[w] = c;
    pthread_mutex_init(&J.mu, NULL);
    if (threads < 1)
        threads = 1;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int t = 0; t < threads; t++)
        pthread_create(&th[t], NULL, scan_worker, &J);
    for (int t = 0; t < threads; t++)
        pthread_join(th[t], NULL);
    free(th);
    pthread_mutex_destroy(&J.mu);
    free(J.rowOff);
    free(J.winContig);
    return 0;
}

/* writeStats (src/KmerDatabase.hpp:935-948): header line, then one row per
 * window in window order, id\tstart\tend\ttotal\tobserved\tvariations\tdistance. */
int orc_write_tsv(const char *path, const orc_seqfile *f, const orc_window *rows, uint32_t W,
                  uint32_t k)
{
    FILE *o = fopen(path, "w");
    if (!o) {
        set_err("Unable to open %s for writing: %s", path, strerror(errno));
        return -1;
    }
    fputs("seqname\tstart\tend\ttotal_kmers\tobserved_kmers\tvariations\tkmer_distance\n", o);
    size_t r = 0;
    for (size_t c = 0; c < f->n; c++) {
        const size_t nw = orc_window_count(f->lens[c], W, k);
        for (size_t w = 0; w < nw; w++, r++)
            fprintf(o, "%s\t%d\t%d\t%d\t%d\t%d\t%d\n", f->ids[c], rows[r].start, rows[r].end,
                    rows[r].total_kmers, rows[r].observed_kmers, rows[r].variations,
                    rows[r].kmer_distance);
    }
    return fclose(o) == 0 ? 0 : -1;
}
