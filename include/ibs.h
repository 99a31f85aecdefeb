/*
 * ibs.h -- C-ABI of the B200 fastibs window scan (libibs.so).
 *
 * Plain C types only: pointers, sizes and the structs below. The library
 * owns every device allocation and all pinned staging; the caller owns the
 * host buffers it passes and the output rows. A handle is used by one host
 * thread at a time. Every call returns an ibs_status; on failure
 * ibs_last_error() (thread-local) holds a one-line message. There is no CPU
 * fallback: without a usable CUDA device the calls return IBS_ERR_CUDA.
 *
 * What it replaces in the reference (GPU-IBS), paths relative to its root:
 *   - the device index (KmcRaIndex load src/gpu/KmcRaIndex.hpp:124-135 +
 *     DeviceKmerIndex upload src/gpu/DeviceKmerIndex.cu:72-142)  -> ibs_open
 *   - the streamed encode+probe engine and its statistics consumer
 *     (EncodeProbeEngine::submit/wait src/gpu/EncodeProbe.cu:941-1022,
 *     :1144-1154; encodeProbeKernel :152-171; BitStats::run
 *     src/gpu/EncodeProbeCore.hpp:338-370 via processReferenceGpu
 *     src/KmerDatabase.hpp:1497-1530)                          -> ibs_scan*
 *   - the panel engine (encodeProbeMultiKernel src/gpu/EncodeProbe.cu:175-193,
 *     KmerPanel::scanRoundGpu src/KmerPanel.hpp:400-439)       -> ibs_scan_panel
 *   - the reference's exceptions "CUDA error in <what>: ..."
 *     (src/gpu/EncodeProbe.cu:15-20)                           -> ibs_status
 */
#ifndef IBS_H
#define IBS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IBS_ABI_VERSION 1

typedef enum ibs_status {
    IBS_OK = 0,
    IBS_ERR_ARG = 1,         /* bad argument (null pointer, W <= k, cap too small) */
    IBS_ERR_IO = 2,          /* file missing / unreadable / short */
    IBS_ERR_FORMAT = 3,      /* not a KMC 3 database this library reads */
    IBS_ERR_CUDA = 4,        /* CUDA runtime error or no usable device */
    IBS_ERR_NOMEM = 5,       /* device or pinned host allocation failed */
    IBS_ERR_UNSUPPORTED = 6, /* k > 64, Quake-mode counters, ... */
    IBS_ERR_CAPACITY = 7,    /* request beyond a fixed capacity */
    IBS_ERR_TIMEOUT = 8,     /* a bounded device wait gave up */
    IBS_ERR_STATE = 9        /* handle in the wrong state for the call */
} ibs_status;

/* One output row: the reference's Window (src/Window.hpp:7-16) minus its id
 * string, which the caller keeps per contig. */
typedef struct ibs_window {
    int32_t start, end, total_kmers, observed_kmers, variations, kmer_distance;
} ibs_window;

typedef struct ibs_table ibs_table;         /* one sample's device-resident k-mer table */
typedef struct ibs_reference ibs_reference; /* a device-resident 2-bit packed reference */

/* Table build options; zero-initialise for the defaults. */
typedef struct ibs_table_opts {
    int device;             /* CUDA device ordinal (default 0) */
    double keys_per_bucket; /* target mean keys per 32 B bucket (0 = ibs_tuning.keys_per_bucket,
                               or 4.0 for a hash table while the tuned format is minimizer lines);
                               for format 8, keys per 128 B line of 8 slots (0 = 4.0) */
    uint32_t force_format;  /* 0 = the tuned default (ibs_tuning.table_format), 1 = B8x32,
                               2 = B6x40, 4 = minimizer lines of B8x32 sectors (16 <= k <= 27),
                               5 = hash buckets, B8x32 or B6x40 by size,
                               6 = minimizer lines of B6x40 sectors (16 <= k <= 31),
                               8 = wide-key lines (33 <= k <= 64, and the only layout there) */
    uint32_t reserved[5];
} ibs_table_opts;

typedef struct ibs_table_info {
    uint32_t k, format, fp_bits, reserved0;
    uint64_t n_keys;         /* k-mers in the table */
    uint64_t n_buckets;      /* 32-byte buckets */
    uint64_t stash_keys;     /* keys that overflowed their bucket */
    uint64_t stash_buckets;
    uint64_t device_bytes;   /* bytes resident on the device */
    double build_seconds;    /* decode + upload + build wall time */
} ibs_table_info;

/* ---- tables -------------------------------------------------------------
 * ibs_open: decode <prefix>.kmc_pre / <prefix>.kmc_suf (KMC 3 formats 0 and
 * 0x200, k <= 64) once and build the device table. Counters are ignored, as
 * the reference's KmcRaIndex strips them (src/gpu/KmcRaIndex.hpp:596-708).
 * Replaces KmcRaIndex(prefix) + DeviceKmerIndex(host, dev, shard) for
 * k <= 32, and for 33 <= k <= 64 the KMC API random-access view that the
 * reference's string path probes (CKMCFile::IsKmer via
 * getStatsFromSequenceLegacy, src/KmerDatabase.hpp:675-708): such a table
 * holds whole 128-bit keys (format 8); the scans (ibs_scan, _async, _packed,
 * _panel), the mapper and ibs_count_present_kmc take it, the joint-table,
 * serving and no-alloc entry points do not (IBS_ERR_ARG / _UNSUPPORTED). */
ibs_status ibs_open(const char *kmc_prefix, const ibs_table_opts *opts, ibs_table **out);

/* Build a table from canonical codes (host or device pointer; duplicates
 * allowed). The k-mer set a KMC database lists, without the file. */
ibs_status ibs_table_from_codes(const uint64_t *codes, uint64_t n, uint32_t k,
                                int codes_on_device, const ibs_table_opts *opts,
                                ibs_table **out);

ibs_status ibs_table_info_get(const ibs_table *t, ibs_table_info *info);

/* A canonical code of a k-mer with 33 <= k <= 64: the 2k-bit code, first
 * base most significant (A=0 C=1 G=2 T=3), as its low and high 64 bits. The
 * reference compares such k-mers as strings (getCanonicalKmersLegacy,
 * src/Utils.hpp:102-125); the order of the codes is the same. */
typedef struct ibs_code128 {
    uint64_t lo, hi;
} ibs_code128;

/* ibs_table_from_codes for 33 <= k <= 64 (a wide-key table, format 8):
 * canonical codes on the host or the device, duplicates allowed (removed on
 * the host before the build). */
ibs_status ibs_table_from_codes128(const ibs_code128 *codes, uint64_t n, uint32_t k,
                                   int codes_on_device, const ibs_table_opts *opts, ibs_table **out);

/* Membership of n wide canonical codes (host array) in a wide-key table,
 * one byte per code: CKMCFile::IsKmer of the string path
 * (src/KmerDatabase.hpp:689-693). ibs_probe / ibs_count_present take the
 * 64-bit codes of k <= 32 tables only. */
ibs_status ibs_probe128(ibs_table *t, const ibs_code128 *codes, uint64_t n, uint8_t *hits);

/* Membership of n canonical codes (host arrays), one byte per code.
 * The probe of KmcRaIndex::probe (src/gpu/KmcRaIndex.hpp:227-235). */
ibs_status ibs_probe(ibs_table *t, const uint64_t *codes, uint64_t n, uint8_t *hits);

/* How many of n canonical codes (host or device array) the table holds.
 * With codes = one database's k-mers and t = another's table this is the
 * intersection size KDBIntersect prints (src/KDBIntersect.cpp:134-233, the
 * probe-and-count of DeviceKmerIndex::probeCountHost). */
ibs_status ibs_count_present(ibs_table *t, const uint64_t *codes, uint64_t n, int codes_on_device,
                             uint64_t *count);

/* The same for every k-mer of a KMC 3 database, decoded on the device: the
 * size of its intersection with the table's k-mer set. IBS_ERR_ARG ("K-mer
 * lengths do not match") when the k differs. Takes wide-key tables (k > 32)
 * too, where KDBIntersect takes its string path (src/KDBIntersect.cpp:386-389). */
ibs_status ibs_count_present_kmc(ibs_table *t, const char *kmc_prefix, uint64_t *count);

void ibs_close(ibs_table *t);

/* Device bytes a table of n_keys k-mers takes (its buckets; the stash of
 * overflowing keys adds about 1% more at the default load). Plans residency
 * the way KmerPanel::imageBytesOf sizes a database (src/KmerPanel.hpp:265-280). */
uint64_t ibs_table_bytes_for(uint64_t n_keys, uint32_t k, const ibs_table_opts *opts);

/* Free and total memory of a device (cudaMemGetInfo), as the reference's
 * DeviceKmerIndex::freeMemory (src/gpu/DeviceKmerIndex.cu:354-367). */
ibs_status ibs_device_memory(int device, uint64_t *free_bytes, uint64_t *total_bytes);

/* ---- references ----------------------------------------------------------
 * Packed layout (the reference's packWindow convention,
 * src/gpu/EncodeProbeCore.hpp:157-186, applied per contig): contig c starts
 * at packed base offset B_c = sum_{c'<c} roundup(len_c', 64); base i of
 * contig c sits at bits 2((B_c+i)%32) of u64 seq word (B_c+i)/32 (A=0 C=1
 * G=2 T=3) and bit (B_c+i)%64 of u64 mask word (B_c+i)/64 is set when the
 * byte is not one of ACGTacgt. ibs_packed_words() gives both array lengths
 * (including one zero word of tail padding each). */
void ibs_packed_words(const uint64_t *lens, uint32_t n_contigs, uint64_t *seq_words,
                      uint64_t *mask_words);

/* Pack ASCII contigs into that layout on the host (the reference's
 * packWindow, src/gpu/EncodeProbeCore.hpp:157-186). */
ibs_status ibs_pack_ascii(const char *const *seqs, const uint64_t *lens, uint32_t n_contigs,
                          uint64_t *seq2bit, uint64_t *nmask, int threads);

/* Upload a packed reference (host pointers) and keep it on the device. */
ibs_status ibs_reference_create(const uint64_t *seq2bit, const uint64_t *nmask,
                                const uint64_t *lens, uint32_t n_contigs, int device,
                                ibs_reference **out);
/* The same from device pointers (copied device-to-device). */
ibs_status ibs_reference_create_device(const uint64_t *seq2bit_dev, const uint64_t *nmask_dev,
                                       const uint64_t *lens, uint32_t n_contigs, int device,
                                       ibs_reference **out);
void ibs_reference_free(ibs_reference *r);

/* A reference straight from FASTA text in host memory (a whole file's bytes;
 * decompress .gz first): the reference's readSequenceFile for FASTA
 * (src/Utils.hpp:170-255) -- lines split on '\n' only, so a '\r' stays
 * and packs as a non-ACGT base; the id is the header line after '>'; a
 * record without sequence is dropped -- with the line-break removal and
 * the packing (packWindow, src/gpu/EncodeProbeCore.hpp:157-186) done on the
 * device. The text goes up through the library's pinned staging (8 x 2
 * slots of 16 MiB per device, allocated by the first call and kept; calls
 * on one device take turns). FASTQ text returns IBS_ERR_UNSUPPORTED (pack it
 * with ibs_pack_ascii); text not starting with '>' or '@' IBS_ERR_FORMAT. */
ibs_status ibs_reference_from_fasta(const char *text, uint64_t n_bytes, int device, ibs_reference **out);
/* Contigs of a reference: count, and each one's length and id (the id
 * string lives as long as the reference; "" when it was built from arrays). */
uint32_t ibs_reference_contig_count(const ibs_reference *r);
ibs_status ibs_reference_contig(const ibs_reference *r, uint32_t i, uint64_t *len, const char **id);
/* The packed arrays back on the host (ibs_packed_words gives the sizes). */
ibs_status ibs_reference_copy_packed(const ibs_reference *r, uint64_t *seq2bit, uint64_t *nmask);

/* ---- mapper ----------------------------------------------------------------
 * fastibsmapper's coverage track (KmerDatabase::produceMapping and
 * getMappingFromSequence, src/KmerDatabase.hpp:774-801, :1067-1204): for
 * each base of each contig, the number of k-mer starts s in [i-k+1, i]
 * whose k bases are ACGT and whose canonical k-mer the table holds.
 * ibs_map_coverage: one byte per base, contigs concatenated (capacity =
 * the sum of the lengths). */
ibs_status ibs_map_coverage(ibs_table *t, ibs_reference *ref, uint8_t *coverage, uint64_t cap);
/* The mapper's output file as text, built on the device: per contig its id,
 * a newline, the coverage values joined by commas, a newline. ids = NULL
 * takes the reference's own ids (ibs_reference_from_fasta); otherwise one
 * per contig. *text is pinned host memory: free it with ibs_map_text_free. */
ibs_status ibs_map_text(ibs_table *t, ibs_reference *ref, const char *const *ids, char **text,
                        uint64_t *n_bytes);
void ibs_map_text_free(char *text);

/* Windows chunkSequences cuts (src/Utils.hpp:296-327): sum over contigs of
 * ceil(len / (W - k)). 0 when W <= k. */
uint64_t ibs_window_count(const uint64_t *lens, uint32_t n_contigs, uint32_t W, uint32_t k);

/* Window starts/ends in output order (host arrays of ibs_window_count).
 * Row coordinates are 32-bit, as the reference's Window::start / end are int
 * (src/Window.hpp:11-12): every call that takes contig lengths (this one,
 * the reference constructors, ibs_reference_from_fasta, ibs_scan_packed,
 * ibs_scan_noalloc) returns IBS_ERR_ARG for a contig longer than 2147483647
 * bases instead of writing wrapped coordinates. */
ibs_status ibs_window_bounds(const uint64_t *lens, uint32_t n_contigs, uint32_t W, uint32_t k,
                             ibs_window *rows, uint64_t cap);

/* ---- scans ---------------------------------------------------------------
 * Every window of every contig of `ref` against table `t`: rows in contig,
 * then window order, bit-identical to the reference CPU path's Window
 * records. W must exceed k (the reference throws, src/Utils.hpp:302-304).
 *
 * ibs_scan: rows to host memory; synchronous. */
ibs_status ibs_scan(ibs_table *t, ibs_reference *ref, uint32_t W, ibs_window *rows,
                    uint64_t cap);

/* ibs_scan_async: rows to device memory `rows_dev`, enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream); returns once enqueued.
 * Scratch is allocated (once per reference and W) before the launch. */
ibs_status ibs_scan_async(ibs_table *t, ibs_reference *ref, uint32_t W, ibs_window *rows_dev,
                          uint64_t cap, void *stream);

/* ibs_scan_packed: the end-to-end call over HOST buffers in the packed
 * layout: uploads the reference in pieces overlapped with the scan and
 * returns the rows in host memory. */
ibs_status ibs_scan_packed(ibs_table *t, const uint64_t *seq2bit, const uint64_t *nmask,
                           const uint64_t *lens, uint32_t n_contigs, uint32_t W,
                           ibs_window *rows, uint64_t cap);

/* Panel: one pass over `ref` against n tables (all of the same k); rows are
 * table-major: rows[i * n_windows + w]. Identical to n single scans
 * (KmerPanel::processReference, src/KmerPanel.hpp:63-234). */
ibs_status ibs_scan_panel(ibs_table *const *tables, uint32_t n_tables, ibs_reference *ref,
                          uint32_t W, ibs_window *rows, uint64_t cap);

/* ---- joint panel tables ----------------------------------------------------
 * One table over up to IBS_PANEL_MAX_SAMPLES samples (the reference's panel
 * limit MAX_DBS, src/gpu/EncodeProbeCore.hpp:291): each 32-byte bucket slot
 * holds a k-mer fingerprint and the mask of the samples that contain it, so
 * a reference position costs one bucket load for the whole panel. Rows of
 * every sample equal its single-sample scan. Replaces the reference's panel
 * engine (encodeProbeMultiKernel src/gpu/EncodeProbe.cu:175-193 over the
 * round's resident DeviceKmerIndex images, src/KmerPanel.hpp:373-439).
 *
 * expected_keys: the number of distinct k-mers over the panel (the union);
 * it sizes the buckets and the overflow stash. Two layouts
 * (opts->force_format): 3 = hash sectors (P5x48: five fingerprints and
 * sample masks per 32-byte sector, any k); 7 = the same sectors on minimizer
 * lines (16 <= k <= 27, at least 2^(2k-28) lines; consecutive positions
 * share 128-byte lines, a full sector spills into its partner sector, then
 * the stash; default load 1.5 keys per sector); 0 = 7 where it applies and its
 * minimum size does not oversize the table, else 3. opts->keys_per_bucket: keys
 * per sector (0 = the tuned panel_keys_per_bucket for 3, 1.5 for 7). Samples are added one at a
 * time (sample i = the i-th call); rows are sample-major:
 * rows[i * n_windows + w]. The scan is a persistent kernel over a work queue
 * of (window, position-range) spans; ibs_panel_table_scan_async captures it
 * (with its work reset and finalizer) as a CUDA graph on the first call for
 * a (reference, W, rows, stream) and replays the graph after that. */
#define IBS_PANEL_MAX_SAMPLES 16
typedef struct ibs_panel_table ibs_panel_table;
ibs_status ibs_panel_table_create(uint32_t k, uint64_t expected_keys, const ibs_table_opts *opts,
                                  ibs_panel_table **out);
ibs_status ibs_panel_table_add_kmc(ibs_panel_table *p, const char *kmc_prefix);
ibs_status ibs_panel_table_add_codes(ibs_panel_table *p, const uint64_t *codes, uint64_t n,
                                     int codes_on_device);
ibs_status ibs_panel_table_info_get(const ibs_panel_table *p, ibs_table_info *info,
                                    uint32_t *n_samples);
/* Sample masks of n codes (bit i = sample i holds the k-mer). */
ibs_status ibs_panel_table_probe(ibs_panel_table *p, const uint64_t *codes, uint64_t n,
                                 uint32_t *masks);
ibs_status ibs_panel_table_scan(ibs_panel_table *p, ibs_reference *ref, uint32_t W,
                                ibs_window *rows, uint64_t cap);
ibs_status ibs_panel_table_scan_async(ibs_panel_table *p, ibs_reference *ref, uint32_t W,
                                      ibs_window *rows_dev, uint64_t cap, void *stream);
void ibs_panel_table_close(ibs_panel_table *p);

/* ---- serving ------------------------------------------------------------------
 * A request loop over one resident reference (no counterpart in the
 * reference, whose CLI scans whole references in batch): requests for
 * different samples and window ranges arrive at any time; sample tables are
 * admitted against a device-memory budget, evicted least-recently-used and
 * reloaded from pinned host copies on a side stream; the loop batches
 * continuously: every launch carries span slices of all runnable requests
 * over their different tables, so a request submitted while others run
 * joins the next launch, and a long request never holds back a short one. A
 * request's rows are exactly the rows of the same windows in a full scan of
 * its sample (alone or in any mix).
 *
 * The server owns a background thread; submit/poll are thread-safe.
 *
 * Batched mode feeds ONE persistent kernel: the loop publishes each
 * iteration's work (span items over the tables, then the rows to fold) as a
 * batch into a ring in pinned host memory; the resident kernel's warps claim
 * the work in order, fold rows straight into pinned host memory and stamp
 * each batch done, so requests that arrive while others run are packed into
 * the same launch. Every device wait is bounded: without new work for
 * idle_exit_us the kernel ends (the next request launches it again), and a
 * fold that waits too long for its batch's scans ends it with a timeout
 * (counted in ibs_server_stats; unfinished batches are published to the
 * next launch). One request per launch (the plain path) launches kernels
 * per request instead. */
typedef struct ibs_server ibs_server;

typedef struct ibs_server_opts {
    int device;
    uint64_t memory_budget;     /* bytes of resident sample tables (0 = 80% of free memory) */
    uint32_t max_spans_per_launch; /* 0 = 1<<15 */
    uint32_t min_spans_per_request; /* per launch, 0 = 16 */
    uint32_t one_request_per_launch; /* 1: no batching (every launch carries one whole request) */
    uint32_t table_format;      /* layout of the single-sample tables the server builds (add_sample_*):
                                   0 = the tuned default (ibs_tuning.table_format: minimizer lines for
                                   large tables), else as ibs_table_opts.force_format */
    double keys_per_bucket;     /* load of those tables (0 = the library default) */
    uint32_t iteration_launches; /* batched mode: 1 = launch kernels per loop iteration instead of
                                    feeding one persistent launch */
    uint32_t idle_exit_us;      /* the persistent launch ends after this long without new work
                                   (0 = 100 ms); the next request launches it again */
} ibs_server_opts;

typedef struct ibs_request_result {
    uint64_t request_id;
    uint32_t sample, contig;
    uint64_t first_window, n_windows; /* window indices within the contig */
    ibs_status status;
    double submit_time, done_time;    /* seconds on the server's clock */
    ibs_window *rows;                 /* n_windows rows, owned by the server until released */
} ibs_request_result;

typedef struct ibs_server_stats {
    uint64_t submitted, completed, launches, spans, probes;
    uint64_t reloads, reload_bytes, evictions;
    uint64_t resident_bytes, resident_tables;
    double busy_seconds;              /* device time of the span launches */
    double latency_p50, latency_p99, latency_max; /* seconds, completed requests */
    uint64_t failed;                  /* completed with a non-OK status (a table reload failed) */
    uint64_t queued, running;         /* waiting for admission / admitted and not yet complete */
    uint64_t scanned;                 /* reference positions the device scanned: a window that several
                                         requests share counts once (probes counts it per request) */
    uint64_t sample_probes;           /* positions x samples the scans answered: a joint-table scan of a
                                         window for three requesting samples counts its positions three
                                         times (two requests of one sample count once) */
    uint64_t persistent_launches;     /* launches of the persistent kernel (batched mode) */
    uint64_t idle_exits;              /* ... that ended after idle_exit_us without new work */
    uint64_t wait_timeouts;           /* ... that ended because a bounded device wait ran out */
    uint64_t replays;                 /* batches published again after their launch ended early */
    uint64_t lookup_failures;         /* published tickets whose batch the kernel did not find (ends it) */
    uint64_t fold_giveups;            /* folds that gave up on stalled spans while a launch was ending */
} ibs_server_stats;

ibs_status ibs_server_create(ibs_reference *ref, uint32_t W, uint32_t k, const ibs_server_opts *opts,
                             ibs_server **out);
/* Registers a sample (its table is built now, copied to pinned host memory
 * for reloads, and kept resident while the budget allows). */
ibs_status ibs_server_add_sample_kmc(ibs_server *s, const char *kmc_prefix, uint32_t *sample_id);
ibs_status ibs_server_add_sample_codes(ibs_server *s, const uint64_t *codes, uint64_t n,
                                       int codes_on_device, uint32_t *sample_id);
/* Registers every sample of a joint panel table; the server keeps its own
 * pinned host image and device copy. The samples get ids first_sample_id ..
 * first_sample_id + n - 1 in the panel's order. Requests for samples of one
 * panel that cover the same windows are scanned together: one bucket load
 * per position answers all of them. With release_panel != 0 the panel's own
 * device table is freed before the server uploads its copy (one copy on the
 * device at a time); the panel handle then only accepts ibs_panel_table_close
 * (other calls return IBS_ERR_STATE). */
ibs_status ibs_server_add_panel(ibs_server *s, ibs_panel_table *panel, int release_panel,
                                uint32_t *first_sample_id);
/* Windows [first_window, first_window + n_windows) of contig `contig`
 * (window i starts at i * (W - k)); n_windows = 0 means to the contig's end. */
ibs_status ibs_server_submit(ibs_server *s, uint32_t sample, uint32_t contig, uint64_t first_window,
                             uint64_t n_windows, uint64_t *request_id);
/* Up to max finished requests (oldest first); timeout_ms < 0 waits for one. */
ibs_status ibs_server_poll(ibs_server *s, ibs_request_result *out, uint32_t max, uint32_t *n_out,
                           int timeout_ms);
/* Frees a polled result's rows. */
void ibs_server_release(ibs_server *s, ibs_request_result *r);
ibs_status ibs_server_stats_get(ibs_server *s, ibs_server_stats *st);
/* Seconds on the server's clock (the clock of submit_time / done_time). */
double ibs_server_now(ibs_server *s);
void ibs_server_close(ibs_server *s);

/* ibs_scan_noalloc: the scan of ibs_scan_async without any memory
 * allocation. No counterpart in the reference. It is for callers that cannot
 * allocate device memory while they scan: a serving process that gave all
 * free device memory to its own pool, a host that keeps its allocations
 * fixed after start-up, or a latency-bound loop in which cudaMalloc (which
 * may synchronize the device) is not acceptable.
 *
 * The caller passes the table, the packed reference in device memory
 * (seq2bit_dev / nmask_dev in the packed layout above), the contig lengths
 * in host memory and the row buffer in device memory; the work is enqueued
 * on `stream` and the call returns. Its scratch (per-contig window table and
 * one 32-byte summary per 4096-position span) is a fixed device array of
 * IBS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * the process exits -- enough for about 4 Gbp of reference at W = 50 kbp. A
 * scan that needs more returns IBS_ERR_CAPACITY before touching the device.
 * All calls on a device share that array: calls whose work overlaps on the
 * GPU (different streams, or different host threads without ordering) race;
 * order them on one stream. The first call on a device looks up the array's
 * device address; make that first call before any stream capture.
 * `lens` is read by an asynchronous host-to-device copy on `stream`: keep it
 * valid and unchanged until the stream has passed the call (when `lens` is
 * pinned the copy may run after the call returns), and, if the call was
 * captured into a CUDA graph, for as long as the graph is replayed (each
 * replay reads it again). Contigs longer than 2147483647 bases return
 * IBS_ERR_ARG (window coordinates are 32-bit). */
#define IBS_NOALLOC_SCRATCH_BYTES (32ull << 20)
ibs_status ibs_scan_noalloc(ibs_table *t, const uint64_t *seq2bit_dev, const uint64_t *nmask_dev,
                            const uint64_t *lens, uint32_t n_contigs, uint32_t W,
                            ibs_window *rows_dev, uint64_t cap, void *stream);

/* ---- tuning -------------------------------------------------------------------
 * Launch shape of the scan kernels and the default table load, process-wide.
 * The committed autotuner (gpu-ibs_b200/python/ibs_b200/autotune.py) sweeps
 * these on the device and records the best in gpu-ibs_b200/tuning/. Zero
 * fields keep the current value. */
typedef struct ibs_tuning {
    uint32_t span_len;         /* k-mer positions per warp task (multiple of 128) */
    uint32_t blocks_in_flight; /* 32-position blocks each lane keeps in flight: 1, 2, 4 or 8 */
    uint32_t block_threads;    /* threads per CTA: 128, 256 or 512 */
    uint32_t ctas_per_sm;      /* resident CTAs per SM the grid is sized for */
    double keys_per_bucket;    /* default load of new tables */
    uint32_t table_format;     /* default format of new tables (0 = automatic, 4 = minimizer buckets) */
    uint32_t panel_pass_mb;    /* joint-table scans probe bucket ranges of at most this many MiB per
                                  pass (random loads over a larger range translate slowly); 0 = 48 GiB */
    uint32_t panel_span_len;   /* positions per work item of the joint-table scan (multiple of 128) */
    uint32_t panel_ctas_per_sm; /* resident CTAs per SM of the persistent joint-table scan (256 threads) */
    double panel_keys_per_bucket; /* default load of new joint tables (keys per 5-slot bucket) */
    uint32_t panel_blocks_in_flight; /* 32-position blocks in flight per lane in that scan: 2 or 4 */
    uint32_t reserved[3];
} ibs_tuning;
/* Fields left 0 keep their value; table_format and panel_pass_mb take
 * 0xffffffff to go back to 0 (automatic / the default). The joint-table
 * fields apply to joint tables created (load) and scans enqueued (launch
 * shape) after the call. */
ibs_status ibs_set_tuning(const ibs_tuning *t);
void ibs_get_tuning(ibs_tuning *t);

/* Last error message of this thread ("" when none). */
const char *ibs_last_error(void);

/* Device count visible to the library (cudaGetDeviceCount; 0 on error). */
int ibs_device_count(void);

/* Kernel launches made by this process's library calls so far. */
uint64_t ibs_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* IBS_H */
