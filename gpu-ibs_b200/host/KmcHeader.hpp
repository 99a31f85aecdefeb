// The header fields of a KMC 3 database's .kmc_pre, read the way the KMC
// API reads them (CKMCFile::ReadParamsFrom_prefix_file_buf,
// KMC/kmc_api/kmc_file.cpp:178-325): version at end-12, the first byte of
// the header offset at end-8, then k, mode, counter size, prefix length,
// signature length (0x200 only), min/max count, total k-mers and the
// both-strands byte (stored negated). What KmerDatabase::printKMCInfo shows.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

namespace ibs_host {

struct KmcInfo {
    uint32_t kmcVersion = 0, kmerLength = 0, mode = 0, counterSize = 0, lutPrefixLength = 0,
             signatureLen = 0, minCount = 0;
    uint64_t maxCount = 0, totalKmers = 0;
    bool bothStrands = false;
};

inline KmcInfo read_kmc_info(const std::string &prefix)
{
    const std::string path = prefix + ".kmc_pre";
    FILE *f = fopen(path.c_str(), "rb");
    if (!f)
        throw std::runtime_error("Could not open KMC database " + prefix);
    auto at = [&](long long off, void *dst, size_t n) {
        if (fseeko(f, off, SEEK_SET) != 0 || fread(dst, 1, n, f) != n) {
            fclose(f);
            throw std::runtime_error("Could not open KMC database " + prefix + " (short .kmc_pre)");
        }
    };
    fseeko(f, 0, SEEK_END);
    const long long size = ftello(f);
    char head[4], tail[4];
    if (size < 24) {
        fclose(f);
        throw std::runtime_error("Could not open KMC database " + prefix + " (short .kmc_pre)");
    }
    at(0, head, 4);
    at(size - 4, tail, 4);
    if (memcmp(head, "KMCP", 4) || memcmp(tail, "KMCP", 4)) {
        fclose(f);
        throw std::runtime_error("Could not open KMC database " + prefix + " (bad marker)");
    }
    KmcInfo k;
    at(size - 12, &k.kmcVersion, 4);
    if (k.kmcVersion != 0 && k.kmcVersion != 0x200) {
        fclose(f);
        throw std::runtime_error("Could not open KMC database " + prefix + " (unsupported version)");
    }
    unsigned char off = 0;
    at(size - 8, &off, 1);
    const long long h = size - ((long long)off + 8);
    if (h < 4) {
        fclose(f);
        throw std::runtime_error("Could not open KMC database " + prefix + " (bad header offset)");
    }
    uint32_t w[7] = {0};
    unsigned char both = 0;
    if (k.kmcVersion == 0x200) {
        at(h, w, 28);
        at(h + 28, &k.totalKmers, 8);
        at(h + 36, &both, 1);
        k.kmerLength = w[0], k.mode = w[1], k.counterSize = w[2], k.lutPrefixLength = w[3];
        k.signatureLen = w[4], k.minCount = w[5], k.maxCount = w[6];
    } else {
        uint32_t hi = 0;
        at(h, w, 24);
        at(h + 24, &k.totalKmers, 8);
        at(h + 32, &both, 1);
        at(h + 33, &hi, 4);
        k.kmerLength = w[0], k.mode = w[1], k.counterSize = w[2], k.lutPrefixLength = w[3];
        k.minCount = w[4];
        k.maxCount = w[5] + ((uint64_t)hi << 32);
    }
    k.bothStrands = !both;
    fclose(f);
    return k;
}

} // namespace ibs_host
