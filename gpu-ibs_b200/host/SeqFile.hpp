// FASTA / FASTQ reading with the reference's semantics
// (readSequenceFile, src/Utils.hpp:170-255; decompressGzip :127-166):
//   - the file type comes from its first byte ('>' FASTA, '@' FASTQ);
//   - lines split on '\n' only (a '\r' stays in ids and sequences);
//   - empty lines are skipped; in FASTQ a line starting with '+' marks the
//     next line as quality, and that check comes before the quality skip;
//   - the id is the whole header line after its first byte;
//   - a record with an empty sequence is dropped;
//   - a truncated or corrupt gzip stream is an error.
#pragma once

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace ibs_host {

struct SequenceFile {
    std::vector<std::string> ids;
    std::vector<std::string> sequences;
};

inline std::string read_gzip(const std::string &path)
{
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f)
        throw std::runtime_error("Failed to open gzip file " + path);
    gzbuffer(f, 1 << 20);
    std::string out;
    std::vector<char> buf(1 << 20);
    for (;;) {
        const int got = gzread(f, buf.data(), (unsigned)buf.size());
        int errnum = Z_OK;
        const char *why = gzerror(f, &errnum);
        if (got < 0 || (errnum != Z_OK && errnum != Z_STREAM_END)) {
            const std::string reason =
                errnum == Z_BUF_ERROR ? "truncated gzip stream" : std::string(why ? why : "read error");
            gzclose(f);
            throw std::runtime_error("Failed to decompress " + path + ": " + reason);
        }
        if (got == 0)
            break;
        out.append(buf.data(), (size_t)got);
    }
    gzclose(f);
    return out;
}

inline std::string read_plain(const std::string &path)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f)
        throw std::runtime_error("Failed to open file " + path);
    fseeko(f, 0, SEEK_END);
    const off_t n = ftello(f);
    fseeko(f, 0, SEEK_SET);
    std::string data((size_t)n, '\0');
    const size_t got = n ? fread(&data[0], 1, (size_t)n, f) : 0;
    fclose(f);
    data.resize(got);
    return data;
}

// A plain file mapped read-only, for readers that only look at its bytes
// (the device FASTA parser copies them through its own pinned staging, so
// the text needs no copy of its own in host memory). Empty when the file
// cannot be mapped; the caller then reads it.
struct MappedFile {
    const char *data = nullptr;
    size_t size = 0;
    explicit MappedFile(const std::string &path)
    {
        const int fd = open(path.c_str(), O_RDONLY);
        if (fd < 0)
            return;
        struct stat st {};
        if (fstat(fd, &st) == 0 && st.st_size > 0) {
            void *p = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (p != MAP_FAILED) {
                madvise(p, (size_t)st.st_size, MADV_SEQUENTIAL | MADV_WILLNEED);
                data = static_cast<const char *>(p);
                size = (size_t)st.st_size;
            }
        }
        close(fd);
    }
    ~MappedFile()
    {
        if (data)
            munmap(const_cast<char *>(data), size);
    }
    MappedFile(const MappedFile &) = delete;
    MappedFile &operator=(const MappedFile &) = delete;
};

inline std::string read_file_text(const std::string &path, bool compressed)
{
    return compressed ? read_gzip(path) : read_plain(path);
}

inline SequenceFile parse_sequence_text(const std::string &data)
{
    if (data.empty())
        throw std::runtime_error("Empty file");
    bool fastq;
    if (data[0] == '>')
        fastq = false;
    else if (data[0] == '@')
        fastq = true;
    else
        throw std::runtime_error("Unknown file type");
    const char idChar = fastq ? '@' : '>';
    SequenceFile out;
    std::string id, seq;
    bool quality = false;
    size_t pos = 0;
    while (pos < data.size()) {
        const char *nl = (const char *)memchr(data.data() + pos, '\n', data.size() - pos);
        const size_t eol = nl ? (size_t)(nl - data.data()) : data.size();
        const char *line = data.data() + pos;
        const size_t len = eol - pos;
        pos = eol + 1;
        if (len == 0)
            continue;
        if (fastq && line[0] == '+') {
            quality = true;
            continue;
        }
        if (quality) {
            quality = false;
            continue;
        }
        if (line[0] == idChar) {
            if (!seq.empty()) {
                out.ids.push_back(std::move(id));
                out.sequences.push_back(std::move(seq));
                id.clear();
                seq.clear();
            }
            id.assign(line + 1, len - 1);
        } else
            seq.append(line, len);
    }
    if (!seq.empty()) {
        out.ids.push_back(std::move(id));
        out.sequences.push_back(std::move(seq));
    }
    return out;
}

inline SequenceFile read_sequence_file(const std::string &path, bool compressed)
{
    return parse_sequence_text(read_file_text(path, compressed));
}

} // namespace ibs_host
