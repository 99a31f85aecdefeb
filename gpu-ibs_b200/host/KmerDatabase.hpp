// KmerDatabase: the reference's single-sample scan interface
// (src/KmerDatabase.hpp: ctor :68-102, getKmerSize, printKMCInfo :54-66,
// processReference :950-1065, writeStats :935-948, writeOutputFile
// :904-931, gpuOptions :222-249) over the B200 scan library (include/ibs.h).
//
// processReference reads the reference (FASTA/FASTQ, optionally gzip), packs
// it 2 bits per base, and scans it on the GPU through ibs_scan_packed; the
// rows are the reference's Window records, written as its TSV. The device
// table is built from the KMC files on the first scan and kept for the next
// references, as the reference keeps its device index. There is no CPU path:
// a failure of the device is an exception, not a fallback.
#pragma once

#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <filesystem>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/ibs.h"
#include "KmcHeader.hpp"
#include "SeqFile.hpp"
#include "Window.hpp"

class KmerDatabase
{
public:
    // The reference's pipeline knobs (src/KmerDatabase.hpp:222-244), kept so
    // command lines and callers that set them still work. Only `gpus` picks
    // anything here (the device: the first of the visible ones); batch size,
    // streams, sync, sorted or hash probing and LUT pinning describe the
    // reference's engine and have no counterpart in this one.
    struct GpuOptions {
        int enable = -1;
        int batchMB = 128;
        int streams = 3;
        bool sync = false;
        bool sortQueries = false;
        bool probeHash = false;
        double hashLoadFactor = 0.6;
        bool pinLut = false;
        int gpus = 0;
        bool noPeer = false;
        bool cpuBatched = false;
        int device = 0; // CUDA device ordinal the tables are built on
    };
    static GpuOptions &gpuOptions()
    {
        static GpuOptions o;
        return o;
    }

    // Header-only open, as the reference's constructor (the table is built
    // on the first scan). Throws std::runtime_error("Could not open KMC
    // database <path>") where the reference prints that line and exits.
    explicit KmerDatabase(std::string sourcePath) : sourcePath(std::move(sourcePath))
    {
        info = ibs_host::read_kmc_info(this->sourcePath);
        kmerSize = info.kmerLength;
        if (kmerSize > 64)
            throw std::runtime_error("k=" + std::to_string(kmerSize) +
                                     " > 64: the device tables hold a k-mer in at most 128 bits");
        if (kmerSize > 32)
            announceWideKeys(kmerSize);
    }

    // k > 32: where the reference takes its string path for the whole process
    // and says so once (routeToStringPath, src/KmerDatabase.hpp:114-124),
    // the scan here builds a wide-key table (128-bit codes) on the device.
    static void announceWideKeys(unsigned k)
    {
        static bool said = false;
        if (said)
            return;
        said = true;
        std::cerr << "[fastibs] k=" << k << " > 32: wide-key device tables (128-bit codes); "
                  << "the --cpu and --probe options do not apply" << std::endl;
    }

    ~KmerDatabase() { releaseGpuIndex(); }
    KmerDatabase(const KmerDatabase &) = delete;
    KmerDatabase &operator=(const KmerDatabase &) = delete;

    unsigned getKmerSize() const { return kmerSize; }
    const std::string &path() const { return sourcePath; }
    const ibs_host::KmcInfo &kmcInfo() const { return info; }

    void printKMCInfo() const
    {
        std::cout << "********** KMC Info **********\n";
        std::cout << "K-mer length: " << info.kmerLength << '\n';
        std::cout << "Mode: " << info.mode << '\n';
        std::cout << "Counter size: " << info.counterSize << '\n';
        std::cout << "LUT prefix length: " << info.lutPrefixLength << '\n';
        std::cout << "Signature length: " << info.signatureLen << '\n';
        std::cout << "Min count: " << info.minCount << '\n';
        std::cout << "Max count: " << info.maxCount << '\n';
        std::cout << "Both strands: " << info.bothStrands << '\n';
        std::cout << "Total k-mers: " << info.totalKmers << '\n';
    }

    // Builds the device table now (processReference does it on first use).
    void initGpuIndex()
    {
        if (table)
            return;
        ibs_table_opts o{};
        o.device = gpuOptions().device;
        const auto t0 = std::chrono::steady_clock::now();
        check(ibs_open(sourcePath.c_str(), &o, &table), "ibs_open");
        ibs_table_info ti{};
        ibs_table_info_get(table, &ti);
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        char msg[200];
        snprintf(msg, sizeof msg,
                 "[gpu] index read+decode+build: %.3f s (%llu k-mers, %.2f GB on device %d)", s,
                 (unsigned long long)ti.n_keys, ti.device_bytes / 1e9, o.device);
        std::cout << msg << std::endl;
    }

    void releaseGpuIndex()
    {
        if (table) {
            ibs_close(table);
            table = nullptr;
        }
    }

    bool gpuActive() const { return table != nullptr; }
    ibs_table *gpuTable() { return table; }

    // A reference read and packed: contig ids, lengths and the packed arrays.
    struct PackedReference {
        std::vector<std::string> ids;
        std::vector<uint64_t> lens;
        std::vector<uint64_t> seq, mask;
        double readSec = 0, packSec = 0;
    };

    static PackedReference readReference(const std::string &refPath)
    {
        const auto t0 = std::chrono::steady_clock::now();
        std::cout << "Reading sequences" << std::endl;
        const bool compressed = refPath.find(".gz") != std::string::npos;
        PackedReference r = packText(ibs_host::read_file_text(refPath, compressed));
        r.readSec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() - r.packSec;
        return r;
    }

    // A reference on the device: FASTA text (plain or gunzipped) is parsed
    // and packed there (ibs_reference_from_fasta); FASTQ is read and packed
    // on the host and uploaded. meta gets the ids and lengths.
    static ibs_reference *loadReference(const std::string &refPath, PackedReference &meta)
    {
        const auto t0 = std::chrono::steady_clock::now();
        std::cout << "Reading sequences" << std::endl;
        const bool compressed = refPath.find(".gz") != std::string::npos;
        if (!compressed) {
            // plain FASTA goes to the device parser straight from the mapped file
            ibs_host::MappedFile mf(refPath);
            if (mf.data && mf.size && mf.data[0] == '>') {
                ibs_reference *dref = nullptr;
                meta = PackedReference();
                const auto t1 = std::chrono::steady_clock::now();
                check(ibs_reference_from_fasta(mf.data, mf.size, gpuOptions().device, &dref),
                      "ibs_reference_from_fasta");
                const uint32_t n = ibs_reference_contig_count(dref);
                for (uint32_t c = 0; c < n; ++c) {
                    uint64_t len = 0;
                    const char *id = nullptr;
                    ibs_reference_contig(dref, c, &len, &id);
                    meta.lens.push_back(len);
                    meta.ids.emplace_back(id);
                }
                meta.readSec = std::chrono::duration<double>(t1 - t0).count();
                meta.packSec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
                return dref;
            }
        }
        std::string text = ibs_host::read_file_text(refPath, compressed);
        const auto t1 = std::chrono::steady_clock::now();
        ibs_reference *dref = nullptr;
        if (!text.empty() && text[0] == '>') {
            meta = PackedReference();
            check(ibs_reference_from_fasta(text.data(), text.size(), gpuOptions().device, &dref),
                  "ibs_reference_from_fasta");
            const uint32_t n = ibs_reference_contig_count(dref);
            for (uint32_t c = 0; c < n; ++c) {
                uint64_t len = 0;
                const char *id = nullptr;
                ibs_reference_contig(dref, c, &len, &id);
                meta.lens.push_back(len);
                meta.ids.emplace_back(id);
            }
            meta.readSec = std::chrono::duration<double>(t1 - t0).count();
            meta.packSec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
            return dref;
        }
        meta = packText(text);
        meta.readSec = std::chrono::duration<double>(t1 - t0).count();
        check(ibs_reference_create(meta.seq.data(), meta.mask.data(), meta.lens.data(),
                                   (uint32_t)meta.lens.size(), gpuOptions().device, &dref),
              "ibs_reference_create");
        return dref;
    }

    // Host reader and packer (FASTQ, and the arrays when a caller wants them).
    static PackedReference packText(const std::string &text)
    {
        PackedReference r;
        const auto t1 = std::chrono::steady_clock::now();
        ibs_host::SequenceFile f = ibs_host::parse_sequence_text(text);
        r.ids = std::move(f.ids);
        std::vector<const char *> ptrs;
        for (const auto &s : f.sequences) {
            r.lens.push_back(s.size());
            ptrs.push_back(s.data());
        }
        uint64_t sw = 0, mw = 0;
        ibs_packed_words(r.lens.data(), (uint32_t)r.lens.size(), &sw, &mw);
        r.seq.assign(sw, 0);
        r.mask.assign(mw, 0);
        check(ibs_pack_ascii(ptrs.data(), r.lens.data(), (uint32_t)r.lens.size(), r.seq.data(),
                             r.mask.data(), (int)std::thread::hardware_concurrency()),
              "ibs_pack_ascii");
        r.packSec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
        return r;
    }

    // Rows of one packed reference as Window records (ids filled in).
    static std::vector<Window> toWindows(const PackedReference &ref, const ibs_window *rows,
                                         uint32_t W, uint32_t k)
    {
        std::vector<Window> out;
        out.reserve(ibs_window_count(ref.lens.data(), (uint32_t)ref.lens.size(), W, k));
        uint64_t r = 0;
        for (size_t c = 0; c < ref.lens.size(); ++c) {
            const uint64_t n = ibs_window_count(&ref.lens[c], 1, W, k);
            for (uint64_t i = 0; i < n; ++i, ++r) {
                Window w;
                w.id = ref.ids[c];
                w.start = rows[r].start;
                w.end = rows[r].end;
                w.totalKmers = rows[r].total_kmers;
                w.observedKmers = rows[r].observed_kmers;
                w.variations = rows[r].variations;
                w.kmerDistance = rows[r].kmer_distance;
                out.push_back(std::move(w));
            }
        }
        return out;
    }

    static void checkWindow(int windowSize, unsigned k)
    {
        if (windowSize <= (int)k)
            throw std::invalid_argument("window size " + std::to_string(windowSize) +
                                        " must be larger than k (" + std::to_string(k) + ")");
    }

    void processReference(const std::string &refPath, const std::string &outPath,
                          int windowSize = 50000)
    {
        auto clock = std::chrono::steady_clock::now();
        auto lap = [&clock]() {
            const auto now = std::chrono::steady_clock::now();
            const double s = std::chrono::duration<double>(now - clock).count();
            clock = now;
            return s;
        };
        initGpuIndex();
        std::cout << "Window size: " << windowSize << std::endl;
        std::cout << "Kmer size: " << kmerSize << std::endl;
        std::cout << "K-mer path: fused GPU encode+probe, sector-bucket table (sm_100a)" << std::endl;
        checkWindow(windowSize, kmerSize);
        const double setupSec = lap();
        PackedReference ref;
        std::unique_ptr<ibs_reference, void (*)(ibs_reference *)> dref(loadReference(refPath, ref),
                                                                        ibs_reference_free);
        lap();
        const uint64_t n = ibs_window_count(ref.lens.data(), (uint32_t)ref.lens.size(),
                                            (uint32_t)windowSize, kmerSize);
        std::cout << "Number of chunks: " << n << std::endl;
        std::cout << "Calculating stats" << std::endl;
        std::vector<ibs_window> rows(n ? n : 1);
        check(ibs_scan(table, dref.get(), (uint32_t)windowSize, rows.data(), n), "ibs_scan");
        const std::vector<Window> stats = toWindows(ref, rows.data(), windowSize, kmerSize);
        const double statsSec = lap();
        std::cout << "Writing stats to file" << std::endl;
        writeStats(outPath, stats);
        const double writeSec = lap();
        std::cout << "Scan phases: setup " << setupSec << " s, read " << ref.readSec
                  << " s, window " << ref.packSec << " s, stats " << statsSec << " s, write "
                  << writeSec << " s" << std::endl;
    }

    // fastibsmapper: the coverage track of every contig (per base, how many
    // of the sample's k-mers cover it) written as "<id>\n<c0,c1,...>\n" per
    // contig (KmerDatabase::produceMapping, src/KmerDatabase.hpp:1067-1204).
    // Probing, the coverage counts and the text are all made on the device.
    void produceMapping(const std::string &refPath, const std::string &outPath)
    {
        auto clock = std::chrono::steady_clock::now();
        auto lap = [&clock]() {
            const auto now = std::chrono::steady_clock::now();
            const double s = std::chrono::duration<double>(now - clock).count();
            clock = now;
            return s;
        };
        initGpuIndex();
        std::cout << "Kmer size: " << kmerSize << std::endl;
        std::cout << "K-mer path: fused GPU encode+probe, coverage and text on the device (sm_100a)"
                  << std::endl;
        PackedReference ref;
        std::unique_ptr<ibs_reference, void (*)(ibs_reference *)> dref(loadReference(refPath, ref),
                                                                        ibs_reference_free);
        lap();
        std::cout << "Calculating mapping" << std::endl;
        std::vector<const char *> ids;
        for (const auto &id : ref.ids)
            ids.push_back(id.c_str());
        char *text = nullptr;
        uint64_t n = 0;
        check(ibs_map_text(table, dref.get(), ids.data(), &text, &n), "ibs_map_text");
        std::unique_ptr<char, void (*)(char *)> textGuard(text, ibs_map_text_free);
        const double probeSec = lap();
        std::cout << "Writing mapping to file" << std::endl;
        writeOutputFile(outPath, [&](std::ofstream &f) { f.write(text, (std::streamsize)n); });
        std::cout << "Mapping phases: read " << ref.readSec << " s, pack " << ref.packSec << " s, probe+serialize "
                  << probeSec << " s, write " << lap() << " s" << std::endl;
    }

    // Output written as "<outPath>.partial" and renamed once complete; a
    // failed open, write or rename throws and leaves no file under the final
    // name (src/KmerDatabase.hpp:899-931).
    template <typename WriteFn>
    static void writeOutputFile(const std::string &outPath, WriteFn write)
    {
        const std::string tmpPath = outPath + ".partial";
        std::error_code ec;
        {
            errno = 0;
            std::ofstream out(tmpPath);
            if (!out.is_open())
                throw std::runtime_error("Unable to open " + tmpPath + " for writing" +
                                         (errno ? std::string(": ") + strerror(errno) : std::string()));
            write(out);
            out.close();
            if (!out) {
                std::filesystem::remove(tmpPath, ec);
                throw std::runtime_error("Writing " + outPath + " failed (disk full or I/O error)");
            }
        }
        std::filesystem::rename(tmpPath, outPath, ec);
        if (ec) {
            std::error_code ignored;
            std::filesystem::remove(tmpPath, ignored);
            throw std::runtime_error("Unable to move " + tmpPath + " to " + outPath + ": " + ec.message());
        }
    }

    static void writeStats(const std::string &outPath, const std::vector<Window> &rows)
    {
        writeOutputFile(outPath, [&rows](std::ofstream &f) {
            f << "seqname\tstart\tend\ttotal_kmers\tobserved_kmers\tvariations\tkmer_distance\n";
            for (const Window &w : rows)
                f << w.id << '\t' << w.start << '\t' << w.end << '\t' << w.totalKmers << '\t'
                  << w.observedKmers << '\t' << w.variations << '\t' << w.kmerDistance << '\n';
        });
    }

    static void check(ibs_status s, const char *what)
    {
        if (s != IBS_OK)
            throw std::runtime_error(std::string(what) + ": " + ibs_last_error());
    }

private:
    std::string sourcePath;
    ibs_host::KmcInfo info;
    unsigned kmerSize = 0;
    ibs_table *table = nullptr;
};
