/*
 * ibs_tools.h -- C-ABI of libibs_tools.so: seeded synthetic references and
 * samples in the shapes of the benchmark workloads, and a KMC 3 database
 * writer. These have no counterpart in the reference, which takes its inputs
 * from FASTA files and the external `kmc` counter; they exist so tests and
 * benchmarks can make inputs of any size without that tool.
 *
 * Generation is counter-based (every base, N run, SNP and k-mer is a pure
 * function of the seed and its index), so the host and device generators
 * produce identical data.
 */
#ifndef IBS_TOOLS_H
#define IBS_TOOLS_H

#include <stdint.h>

#include "ibs.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ibs_synth_ref_spec {
    uint64_t seed;
    uint32_t n_contigs;
    uint32_t reserved0;
    const uint64_t *lens;     /* contig lengths */
    double n_frac;            /* fraction of bases covered by N runs (approximate) */
    uint32_t n_run_min, n_run_max;
    double lower_frac;        /* fraction of bases in lowercase runs (FASTA text only) */
    uint32_t lower_run_min, lower_run_max;
} ibs_synth_ref_spec;

typedef struct ibs_synth_sample_spec {
    uint64_t seed;
    uint32_t k;
    uint32_t n_classes;        /* 1..4 SNP-divergence classes */
    uint64_t block_len;        /* divergence / presence block length in bases */
    double class_rate[4];      /* SNP probability per base of each class */
    double class_prob[4];      /* probability of each class per block */
    double present_frac;       /* probability that a block is present (1 = all) */
    double random_frac;        /* extra random k-mers, as a fraction of total reference length */
    uint32_t n_intro;          /* introgression blocks (override the class rate) */
    uint32_t reserved0;
    const uint32_t *intro_contig;
    const uint64_t *intro_start, *intro_len;
    double intro_rate;
} ibs_synth_sample_spec;

/* N runs of every contig as (contig, start, length) triples; returns the
 * count (call with cap 0 to size). */
uint64_t ibs_synth_n_runs(const ibs_synth_ref_spec *spec, uint32_t *contig, uint64_t *start,
                          uint64_t *len, uint64_t cap);

/* The reference in the packed layout of ibs.h (ibs_packed_words sizes the
 * arrays); on_device != 0: the arrays are device pointers. */
ibs_status ibs_synth_reference(const ibs_synth_ref_spec *spec, uint64_t *seq2bit, uint64_t *nmask,
                               int on_device);

/* The reference as ASCII (ACGT, N in runs, lowercase runs), one contig. */
ibs_status ibs_synth_contig_ascii(const ibs_synth_ref_spec *spec, uint32_t contig, char *out);

/* FASTA file of the reference: ">" + names[c] (or "chr<c+1>"), line_width
 * bases per line. */
ibs_status ibs_synth_write_fasta(const ibs_synth_ref_spec *spec, const char *path,
                                 const char *const *names, uint32_t line_width);

/* The sample's canonical k-mers (duplicates possible; order unspecified on
 * the device). With codes == NULL only *n_out (an upper bound of the count
 * when on_device, exact on the host) is returned. The packed reference comes
 * from ibs_synth_reference (host or device, as on_device says). */
ibs_status ibs_synth_sample_codes(const ibs_synth_ref_spec *ref, const ibs_synth_sample_spec *smp,
                                  const uint64_t *seq2bit, const uint64_t *nmask, int on_device,
                                  uint64_t *codes, uint64_t cap, uint64_t *n_out);

/* KMC 3 database writer. Layout as the KMC API reads it: .kmc_pre = "KMCP",
 * bin-major LUT (n_bins * 4^p cumulative u64 + guard), signature map
 * (4^sig_len + 1 u32), a 64-byte header ending in the version, the header
 * offset, "KMCP"; .kmc_suf = "KMCS", records (suffix bytes big-endian,
 * counter little-endian), "KMCS". version 0 writes the KMC1 layout (one LUT,
 * no signature map). Codes are sorted and deduplicated; counters are
 * 2 + (hash of the code) % 254, capped by the counter width. */
typedef struct ibs_kmc_spec {
    uint32_t k, p, sig_len, n_bins;
    uint32_t counter_size;  /* bytes per counter, 0..4 */
    uint32_t version;       /* 0x200 (KMC2 layout) or 0 (KMC1 layout) */
    uint32_t min_count, max_count;
    uint64_t count_seed;
} ibs_kmc_spec;

ibs_status ibs_kmc_write(const char *prefix, const ibs_kmc_spec *spec, const uint64_t *codes,
                         uint64_t n, int on_device, uint64_t *n_written);

/* The same for 33 <= k <= 64: 128-bit canonical codes from host memory
 * (ibs_code128 of ibs.h); records carry (k - p) / 4 suffix bytes. */
ibs_status ibs_kmc_write128(const char *prefix, const ibs_kmc_spec *spec, const ibs_code128 *codes,
                            uint64_t n, uint64_t *n_written);

/* Random 32-byte-sector read rate of this device over a buffer of `bytes`
 * (uniformly random sector indexes, 4 loads in flight per thread): the
 * ceiling of a scan that reads one random sector per probe. */
ibs_status ibs_random_sector_rate(uint64_t bytes, double *sectors_per_s);

/* Sorted unique canonical codes in place (host); returns the new length. */
uint64_t ibs_sort_unique_host(uint64_t *codes, uint64_t n, int threads);

const char *ibs_tools_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
