// KDBIntersect: the size of the intersection of two KMC 3 databases (the
// reference's tool, src/KDBIntersect.cpp), on the B200.
//
//   KDBIntersect <kDB1Path> <kDB2Path>
//
// Same command line, folder resolution, messages and exit status: the count
// alone on stdout and exit 0; one error line on stderr and exit 1 for a bad
// command line or database. As in the reference, the database with more
// k-mers (by the headers; on a tie the larger .kmc_pre in whole MB, then the
// second argument) becomes the probed structure and the other one is
// enumerated (src/KDBIntersect.cpp:360-375). Here the larger one is decoded
// into a device table (ibs_open), the smaller one is decoded on the device
// and every one of its k-mers is probed there, with only the count coming
// back (ibs_count_present_kmc).
#include <chrono>
#include <cstdio>
#include <filesystem>
#include <iostream>
#include <string>

#include "ibs.h"

#include "CliInput.hpp"
#include "KmcHeader.hpp"

namespace fs = std::filesystem;
using std::cerr;
using std::cout;
using std::endl;
using std::string;

#ifndef IBS_VERSION
#define IBS_VERSION "1.0"
#endif

namespace {

void usage(const char *argv0)
{
    cout << "\nK-mer Database Intersection Tool\n"
         << "----------------------------------\n"
         << "Usage:\n"
         << "  " << argv0 << " <kDB1Path> <kDB2Path>\n\n"
         << "Arguments:\n"
         << "  <kDB1Path>     Path to the first KMC database directory\n"
         << "  <kDB2Path>     Path to the second KMC database directory\n\n"
         << "Description:\n"
         << "  Prints how many k-mers the two KMC databases have in common. The larger\n"
         << "  database (by k-mer count) is decoded into a device table and every k-mer of\n"
         << "  the smaller one is probed against it on the GPU.\n\n"
         << "Notes:\n"
         << "  - The databases must have the same k-mer size (k <= 64; k > 32 builds a wide-key table).\n"
         << "  - Exit status: 0 with the count on stdout; 1 on a bad command line or\n"
         << "    database (one error line on stderr).\n"
         << "  - FASTIBS_GPU_DEVICE=N picks the CUDA device (default 0).\n"
         << "  - --version prints the version and exits.\n\n";
}

int run(int argc, char **argv)
{
    for (int a = 1; a < argc; a++)
        if (string(argv[a]) == "--version") {
            cout << "KDBIntersect (GPU-IBS, B200 scan) " << IBS_VERSION << ", sm_100a build" << endl;
            return 0;
        }
    bool help = false;
    for (int a = 1; a < argc; a++)
        if (string(argv[a]) == "-h" || string(argv[a]) == "--help")
            help = true;
    if (argc != 3 || help) {
        usage(argv[0]);
        return help ? 0 : 1;
    }
    string dir1 = argv[1], dir2 = argv[2];
    ibs_cli::trim_slash(dir1);
    ibs_cli::trim_slash(dir2);
    string db1, db2;
    if (!ibs_cli::resolve_database(dir1, db1) || !ibs_cli::resolve_database(dir2, db2))
        return 1;
    ibs_host::KmcInfo h1, h2;
    try {
        h1 = ibs_host::read_kmc_info(db1);
        h2 = ibs_host::read_kmc_info(db2);
    } catch (const std::exception &e) {
        cerr << "Error: " << e.what() << endl;
        return 1;
    }
    if (h1.kmerLength != h2.kmerLength) {
        cerr << "Error: K-mer lengths do not match" << endl;
        return 1;
    }
    if (h1.kmerLength > 64) {
        cerr << "Error: k = " << h1.kmerLength << " is above 64, which this program does not handle" << endl;
        return 1;
    }
    // small (enumerated) = db1, big (probed) = db2 after the reference's rule
    if (h1.totalKmers != h2.totalKmers) {
        if (h1.totalKmers > h2.totalKmers)
            std::swap(db1, db2);
    } else {
        std::error_code ec;
        const uint64_t mb1 = fs::file_size(db1 + ".kmc_pre", ec) / 1024 / 1024;
        const uint64_t mb2 = fs::file_size(db2 + ".kmc_pre", ec) / 1024 / 1024;
        if (mb1 > mb2)
            std::swap(db1, db2);
    }
    ibs_table_opts o{};
    if (const char *d = getenv("FASTIBS_GPU_DEVICE"))
        o.device = atoi(d);
    const auto t0 = std::chrono::steady_clock::now();
    ibs_table *table = nullptr;
    if (ibs_open(db2.c_str(), &o, &table) != IBS_OK) {
        cerr << "Error: " << ibs_last_error() << endl;
        return 1;
    }
    const auto t1 = std::chrono::steady_clock::now();
    uint64_t count = 0;
    const ibs_status s = ibs_count_present_kmc(table, db1.c_str(), &count);
    ibs_close(table);
    if (s != IBS_OK) {
        cerr << "Error: " << ibs_last_error() << endl;
        return 1;
    }
    const auto t2 = std::chrono::steady_clock::now();
    auto sec = [](auto a, auto b) { return std::chrono::duration<double>(b - a).count(); };
    char msg[256];
    snprintf(msg, sizeof msg, "[gpu] intersect: table of %s in %.3f s, %s probed in %.3f s", db2.c_str(),
             sec(t0, t1), db1.c_str(), sec(t1, t2));
    cerr << msg << endl;
    cout << count << endl;
    if (!cout) {
        cerr << "Error: writing the count to standard output failed" << endl;
        return 1;
    }
    return 0;
}

} // namespace

int main(int argc, char **argv)
{
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        cerr << "Error: " << e.what() << endl;
        return 1;
    }
}
