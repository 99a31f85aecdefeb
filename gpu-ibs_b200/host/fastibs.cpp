// fastibs: the reference's command line (src/FastIBS.cpp, src/GpuCli.hpp,
// src/CliInput.hpp) over the B200 scan.
//
//   fastibs <sourcePath> <referencePath> <resultsFolder> <windowSize> [options]
//
// Same positional arguments, output names (<db>_v_<ref>_<W>.tsv with the
// reference name cut at "_genome"), skip-if-exists rule, per-reference error
// log (log.txt, exit status 1) and panel options (--db, --db-list,
// --resident). The reference's engine knobs are accepted; those with no
// meaning for this engine are ignored, and --cpu / --probe=batched (the
// reference's CPU paths, which this program does not have) say so and scan on
// the GPU, whose rows are identical.
#include <algorithm>
#include <cerrno>
#include <climits>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "CliInput.hpp"
#include "GpuCli.hpp"
#include "KmerDatabase.hpp"
#include "KmerPanel.hpp"

namespace fs = std::filesystem;
using std::cerr;
using std::cout;
using std::endl;
using std::string;
using std::vector;

#ifndef IBS_VERSION
#define IBS_VERSION "1.0"
#endif

namespace {

using ibs_cli::list_references;
using ibs_cli::parse_int;
using ibs_cli::log_reference_error;
using ibs_cli::prepare_results;
using ibs_cli::resolve_database;
using ibs_cli::strip_gz;
using ibs_cli::trim_slash;

struct PanelOptions {
    vector<string> dbs;
    string listFile;
    int resident = 0;
};


string reference_name(const string &filename)
{
    const size_t pos = filename.find("_genome");
    return pos == string::npos ? filename : filename.substr(0, pos);
}


void window_too_small(int W, unsigned k)
{
    cerr << "Error: <windowSize> " << W << " must be larger than the database's k (" << k
         << "): consecutive windows overlap by k bases, so W > k is required" << endl;
}

void usage(const char *argv0)
{
    cout << "\nFastIBS - IBS Distance Calculator (B200 scan)\n"
         << "----------------------------------\n"
         << "Usage:\n"
         << "  " << argv0 << " <sourcePath> <referencePath> <resultsFolder> <windowSize> [options]\n\n"
         << "Arguments:\n"
         << "  <sourcePath>     Path to folder with KMC dataset\n"
         << "  <referencePath>  Path to folder with reference genomes (FASTA)\n"
         << "  <resultsFolder>  Path to folder for storing output results\n"
         << "  <windowSize>     Length of the sequence window for IBS calculation\n"
         << "                   (integer larger than k, e.g., 50000)\n\n"
         << "Options:\n"
         << "  --gpu            Scan on the GPU (the only path of this program)\n"
         << "  --device=N       CUDA device ordinal (default 0)\n"
         << "  --cpu, --probe=batched\n"
         << "                   The reference's CPU paths: not in this program; the scan runs\n"
         << "                   on the GPU with identical rows\n"
         << "  --batch-mb=N --streams=N --sync --sort-queries --probe=bs|hash --hash-lf=F\n"
         << "  --pin-lut --gpus=N|all --no-peer\n"
         << "                   The reference's engine knobs: accepted, no effect here\n"
         << "  -h, --help       Print this text and exit\n"
         << "  --version        Print the version and exit\n\n"
         << "Panel mode (several databases, one reference pass):\n"
         << "  --db=<path>      Another KMC dataset folder to scan in the same pass\n"
         << "  --db-list=<file> A file with one dataset folder per line (# comments)\n"
         << "  --resident=N     At most N databases resident at once (default: as many as fit)\n\n"
         << "Output:\n"
         << "  A tab-delimited file per database and reference: seqname, start, end,\n"
         << "  total_kmers, observed_kmers, variations, kmer_distance\n\n";
}

bool parse_options(int argc, char **argv, int first, PanelOptions &panel)
{
    for (int a = first; a < argc; a++) {
        const string arg = argv[a];
        const int g = ibs_cli::parse_gpu_flag(arg);
        if (g < 0)
            return false;
        if (g > 0)
            continue;
        if (arg.rfind("--db=", 0) == 0 && arg.size() > 5)
            panel.dbs.push_back(arg.substr(5));
        else if (arg.rfind("--db-list=", 0) == 0 && arg.size() > 10)
            panel.listFile = arg.substr(10);
        else if (arg.rfind("--resident=", 0) == 0) {
            if (!ibs_cli::int_option(arg, 11, panel.resident, 0))
                return false;
        } else {
            cerr << "Unknown option: " << arg << endl;
            return false;
        }
    }
    return true;
}

int run_single(const string &dbDir, const vector<fs::path> &refs, const string &refPath,
               const string &results, int W)
{
    string prefix;
    if (!resolve_database(dbDir, prefix))
        return 1;
    const string database = fs::path(dbDir).filename().string();
    cout << "****Database: " << database << endl;
    cout << "Using sourcePath: " << prefix << endl;
    cout << "Using referencePath: " << refPath << endl;
    cout << "Using resultsFolder: " << results << endl;
    std::unique_ptr<KmerDatabase> db;
    try {
        db = std::make_unique<KmerDatabase>(prefix);
    } catch (const std::exception &e) {
        cerr << "Error: " << e.what() << endl;
        return 1;
    }
    db->printKMCInfo();
    cout << "********************************************" << endl;
    if (W <= (int)db->getKmerSize()) {
        window_too_small(W, db->getKmerSize());
        return 1;
    }
    if (!prepare_results(results))
        return 1;
    int failed = 0;
    for (const auto &ref : refs) {
        const string refName = reference_name(ref.filename().string());
        cout << "Processing reference: " << refName << endl;
        const string out = results + "/" + database + "_v_" + refName + "_" + std::to_string(W) + ".tsv";
        if (fs::exists(out)) {
            cout << "File already exists, skipping..." << endl;
            continue;
        }
        try {
            db->processReference(ref.string(), out, W);
        } catch (const std::exception &e) {
            failed++;
            log_reference_error(refName, e);
        }
    }
    if (failed)
        cerr << failed << " reference(s) failed; see log.txt" << endl;
    return failed ? 1 : 0;
}

int run_panel(vector<string> dirs, const vector<fs::path> &refs, const string &refPath,
              const string &results, int W, int resident)
{
    vector<string> prefixes, names;
    for (string &dir : dirs) {
        trim_slash(dir);
        const string name = fs::path(dir).filename().string();
        if (std::find(names.begin(), names.end(), name) != names.end()) {
            cerr << "Error: two panel databases are named " << name
                 << " (their outputs would share a file name)" << endl;
            return 1;
        }
        string prefix;
        if (!resolve_database(dir, prefix))
            return 1;
        names.push_back(name);
        prefixes.push_back(prefix);
    }
    // k > 32: no joint table holds such k-mers, so the databases are scanned
    // one at a time, writing the files a panel would (src/FastIBS.cpp:155-180);
    // every member's k is read first, as a panel shares one k
    try {
        const uint32_t k = ibs_host::read_kmc_info(prefixes[0]).kmerLength;
        for (size_t i = 1; i < prefixes.size(); i++) {
            const uint32_t ki = ibs_host::read_kmc_info(prefixes[i]).kmerLength;
            if (ki != k) {
                cerr << "Error: KmerPanel: " << names[i] << " has k=" << ki << " but " << names[0] << " has k=" << k
                     << "; a panel shares one k" << endl;
                return 1;
            }
        }
        if (k > 32) {
            cout << "[panel] k=" << k << " > 32 has no panel path; scanning the " << dirs.size()
                 << " databases one at a time" << endl;
            int status = 0;
            for (const string &dir : dirs)
                status |= run_single(dir, refs, refPath, results, W);
            return status;
        }
    } catch (const std::exception &e) {
        cerr << "Error: " << e.what() << endl;
        return 1;
    }
    cout << "****Panel: " << dirs.size() << " databases" << endl;
    for (size_t i = 0; i < prefixes.size(); i++)
        cout << "  " << names[i] << " (" << prefixes[i] << ")" << endl;
    cout << "Using referencePath: " << refPath << endl;
    cout << "Using resultsFolder: " << results << endl;
    std::unique_ptr<KmerPanel> panel;
    try {
        panel = std::make_unique<KmerPanel>(prefixes, names, resident);
    } catch (const std::exception &e) {
        cerr << "Error: " << e.what() << endl;
        return 1;
    }
    if (W <= (int)panel->kmerSize()) {
        window_too_small(W, panel->kmerSize());
        return 1;
    }
    if (!prepare_results(results))
        return 1;
    int failed = 0;
    for (const auto &ref : refs) {
        const string refName = reference_name(ref.filename().string());
        cout << "Processing reference: " << refName << endl;
        vector<string> outs(panel->size());
        size_t pending = 0;
        for (size_t i = 0; i < panel->size(); i++) {
            outs[i] = results + "/" + panel->name(i) + "_v_" + refName + "_" + std::to_string(W) + ".tsv";
            if (fs::exists(outs[i])) {
                cout << "File already exists for " << panel->name(i) << ", skipping..." << endl;
                outs[i].clear();
            } else
                pending++;
        }
        if (!pending)
            continue;
        try {
            panel->processReference(ref.string(), outs, W);
        } catch (const std::exception &e) {
            failed++;
            log_reference_error(refName, e);
        }
    }
    if (failed)
        cerr << failed << " reference(s) failed; see log.txt" << endl;
    return failed ? 1 : 0;
}

int run(int argc, char **argv)
{
    for (int a = 1; a < argc; a++)
        if (string(argv[a]) == "--version") {
            cout << "fastibs (GPU-IBS, B200 scan) " << IBS_VERSION << ", sm_100a build" << endl;
            return 0;
        }
    for (int a = 1; a < argc; a++)
        if (string(argv[a]) == "-h" || string(argv[a]) == "--help") {
            usage(argv[0]);
            return 0;
        }
    if (argc < 5) {
        usage(argv[0]);
        return 1;
    }
    string source = argv[1], refPath = argv[2], results = argv[3];
    int W = 0;
    if (!parse_int(argv[4], 1, W)) {
        cerr << "Invalid <windowSize>: " << argv[4] << " (expected a positive integer)" << endl;
        usage(argv[0]);
        return 1;
    }
    PanelOptions panel;
    if (!parse_options(argc, argv, 5, panel)) {
        usage(argv[0]);
        return 1;
    }
    trim_slash(source);
    trim_slash(refPath);
    trim_slash(results);
    vector<string> dirs = panel.dbs;
    if (!panel.listFile.empty()) {
        std::ifstream list(panel.listFile);
        if (!list) {
            cerr << "Error: cannot open --db-list file: " << panel.listFile << endl;
            return 1;
        }
        string line;
        while (std::getline(list, line)) {
            const size_t a = line.find_first_not_of(" \t\r");
            if (a == string::npos || line[a] == '#')
                continue;
            const size_t b = line.find_last_not_of(" \t\r");
            dirs.push_back(line.substr(a, b - a + 1));
        }
    }
    vector<fs::path> refs;
    if (!list_references(refPath, refs))
        return 1;
    if (!dirs.empty()) {
        dirs.insert(dirs.begin(), source);
        return run_panel(dirs, refs, refPath, results, W, panel.resident);
    }
    return run_single(source, refs, refPath, results, W);
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
