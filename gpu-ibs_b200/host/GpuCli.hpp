// The engine options the reference's GPU tools accept (src/GpuCli.hpp:17-71),
// shared by fastibs and fastibsmapper. Those that steer a part of the
// reference's engine this library does not have are accepted and ignored;
// --cpu / --probe=batched (the reference's CPU paths) warn and run on the
// GPU, whose results are identical.
#pragma once

#include <cerrno>
#include <climits>
#include <cstdlib>
#include <iostream>
#include <string>

#include "KmerDatabase.hpp"

namespace ibs_cli {

inline bool parse_int(const std::string &text, int lo, int &out)
{
    const char *s = text.c_str();
    char *end = nullptr;
    errno = 0;
    const long long v = std::strtoll(s, &end, 10);
    if (end == s || *end != '\0' || errno == ERANGE || v < lo || v > INT_MAX)
        return false;
    out = (int)v;
    return true;
}

// "--name=<int>" with the value starting at n; false after an error line.
inline bool int_option(const std::string &arg, size_t n, int &out, int lo = 1)
{
    if (parse_int(arg.substr(n), lo, out))
        return true;
    std::cerr << "Invalid value for option: " << arg << " (expected an integer >= " << lo << ")" << std::endl;
    return false;
}

// 1: a GPU option, applied; 0: not one of them; -1: a bad value (an error
// line is printed).
inline int parse_gpu_flag(const std::string &arg)
{
    auto &o = KmerDatabase::gpuOptions();
    if (arg == "--gpu")
        o.enable = 1;
    else if (arg == "--cpu" || arg == "--probe=batched") {
        o.enable = 0;
        std::cerr << "Warning: " << arg << " selects the reference's CPU path, which this program does "
                  << "not have; running on the GPU (identical results)" << std::endl;
    } else if (arg == "--sync")
        o.sync = true;
    else if (arg.rfind("--batch-mb=", 0) == 0)
        return int_option(arg, 11, o.batchMB) ? 1 : -1;
    else if (arg.rfind("--streams=", 0) == 0)
        return int_option(arg, 10, o.streams) ? 1 : -1;
    else if (arg == "--gpus=all")
        o.gpus = 0;
    else if (arg == "--gpus=0") {
        std::cerr << "Invalid value for option: --gpus=0 (use --gpus=all for every device, --cpu for none)"
                  << std::endl;
        return -1;
    } else if (arg.rfind("--gpus=", 0) == 0)
        return int_option(arg, 7, o.gpus) ? 1 : -1;
    else if (arg.rfind("--device=", 0) == 0)
        return int_option(arg, 9, o.device, 0) ? 1 : -1;
    else if (arg == "--no-peer")
        o.noPeer = true;
    else if (arg == "--sort-queries")
        o.sortQueries = true;
    else if (arg == "--probe=bs" || arg == "--probe=hash")
        o.probeHash = arg == "--probe=hash";
    else if (arg == "--pin-lut")
        o.pinLut = true;
    else if (arg.rfind("--hash-lf=", 0) == 0) {
        double v = 0;
        try {
            size_t used = 0;
            v = std::stod(arg.substr(10), &used);
            if (used != arg.size() - 10)
                v = 0;
        } catch (const std::exception &) {
            v = 0;
        }
        if (v < 0.1 || v > 0.95) {
            std::cerr << "Invalid value for option: " << arg << " (expected 0.1 .. 0.95)" << std::endl;
            return -1;
        }
        o.hashLoadFactor = v;
    } else
        return 0;
    return 1;
}

} // namespace ibs_cli
