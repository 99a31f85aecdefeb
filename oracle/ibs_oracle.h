/*
 * CPU oracle for the fastibs window scan -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's CPU scan path (GPU-IBS, the
 * CPU-BATCHED/CPU-OPT statistics loop), used by the tests, by smoke() and
 * by bench.py's cpu_baseline leg as the checker. Nothing in the product
 * (the CUDA library, the C-ABI, the host facade or the CLI) links, loads
 * or calls this code.
 *
 * Parity is pinned against the reference's own fastibs binary built from
 * its sources (oracle/build_ref.sh -> oracle/_ref/fastibs): the committed
 * golden TSVs under tests/golden/ were produced by that binary and are
 * compared byte for byte with this oracle's output by tests/test_oracle.py.
 */
#ifndef IBS_ORACLE_H
#define IBS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One output row (src/Window.hpp:7-16, minus the id string). */
typedef struct orc_window {
    int32_t start, end, total_kmers, observed_kmers, variations, kmer_distance;
} orc_window;

/* ---- FASTA / FASTQ (src/Utils.hpp:170-255) ---------------------------- */
typedef struct orc_seqfile orc_seqfile;
/* Returns NULL on error; orc_error() says why. compressed != 0 reads gzip. */
orc_seqfile *orc_read_sequence_file(const char *path, int compressed);
size_t orc_seqfile_count(const orc_seqfile *f);
const char *orc_seqfile_id(const orc_seqfile *f, size_t i);
const char *orc_seqfile_seq(const orc_seqfile *f, size_t i, size_t *len);
void orc_seqfile_free(orc_seqfile *f);

/* ---- KMC random-access index (src/gpu/KmcRaIndex.hpp:124-750) --------- */
typedef struct orc_index orc_index;
orc_index *orc_index_open(const char *prefix);
void orc_index_close(orc_index *ix);
/* k, p, sigLen, suffixBytes, counterBytes, nBins; totalKmers via *total */
void orc_index_params(const orc_index *ix, uint32_t out[6], uint64_t *total);
/* Membership of one canonical code (src/gpu/ProbeCore.hpp:113-129). */
int orc_probe(const orc_index *ix, uint64_t code);
void orc_probe_many(const orc_index *ix, const uint64_t *codes, size_t n, uint8_t *hits);
/* Every k-mer of the index in on-disk order (KmcRaIndex::forEachKmer,
 * src/gpu/KmcRaIndex.hpp:169-173, :446-460); returns the count written. */
size_t orc_index_list(const orc_index *ix, uint64_t *codes, size_t cap);
uint32_t orc_signature(const orc_index *ix, uint64_t code);
/* orc_probe / orc_index_list answer 0 for k > 32 indexes, which take these.
 * k > 32 (the reference's string path, KMC API CKMCFile::IsKmer): membership
 * of one 128-bit canonical code given as its low and high words, and the
 * listing as two word arrays. */
int orc_probe128(const orc_index *ix, uint64_t lo, uint64_t hi);
size_t orc_index_list128(const orc_index *ix, uint64_t *lo, uint64_t *hi, size_t cap);

/* ---- codec (src/KmerCodec.hpp:38-61) ---------------------------------- */
/* Canonical codes of all valid positions, in order; returns the count. */
size_t orc_canonical_codes(const char *seq, size_t len, uint32_t k, uint64_t *codes);
/* k > 32: canonical k-mers of the string path (src/Utils.hpp:102-125) as
 * 128-bit codes split into low and high words. */
size_t orc_canonical_codes128(const char *seq, size_t len, uint32_t k, uint64_t *lo, uint64_t *hi);

/* ---- windows (src/Utils.hpp:296-327) ---------------------------------- */
/* Number of windows chunkSequences cuts from a contig of `len` bases. */
size_t orc_window_count(size_t len, uint32_t W, uint32_t k);

/* ---- the scan --------------------------------------------------------- */
/* Statistics of every window of one contig against the index (or, with
 * ix == NULL, against the synthetic predicate pred_mul: code*pred_mul >> 61
 * == 0, the hit rule of the reference's tests/phase2_test.cpp:219-220).
 * rows must hold orc_window_count(len, W, k) entries. Returns 0 on success. */
int orc_scan_contig(const orc_index *ix, const char *seq, size_t len, uint32_t W,
                    uint32_t k, orc_window *rows);
/* The same over several contigs with `threads` worker threads (contig and
 * window order kept; rows laid out contig after contig). */
int orc_scan_contigs(const orc_index *ix, const char *const *seqs, const size_t *lens,
                     size_t n, uint32_t W, uint32_t k, int threads, orc_window *rows);
/* Statistics over a caller-supplied hit rule: hits[i] answers the i-th
 * canonical code of the window (used to pin the statistics loop alone). */
void orc_stats_from_hits(const uint8_t *hits, size_t n, uint32_t k, orc_window *row);

/* The TSV the reference writes (src/KmerDatabase.hpp:935-948) for one
 * sequence file: returns 0 on success. */
int orc_write_tsv(const char *path, const orc_seqfile *f, const orc_window *rows,
                  uint32_t W, uint32_t k);

const char *orc_error(void);

#ifdef __cplusplus
}
#endif
#endif
