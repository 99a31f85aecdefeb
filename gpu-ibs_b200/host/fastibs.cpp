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
// reference's CPU paths, which this build does not have) say so and scan on
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

using ibs_cli::resolve_database;
using ibs_cli::trim_slash;

struct PanelOptions {
    vector<string> dbs;
    string listFile;
    int resident = 0;
};

bool parse_int(const string &text, int lo, int &out)
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

string reference_name(const string &filename)
{
    const size_t pos = filename.find("_genome");
    return pos == string::npos ? filename : filename.substr(0, pos);
}

void log_reference_error(const string &refName, const std::exception &e)
{
    cerr << "Error processing reference " << refName << ": " << e.what() << " (also in log.txt)"
         << endl;
    std::ofstream log("log.txt", std::ios::app);
    if (log.is_open())
        log << "Error processing reference: " << refName << endl << e.what() << endl;
    else
        cout << "Unable to open log file." << endl;
}

string strip_gz(const string &f)
{
    return f.size() > 3 && f.compare(f.size() - 3, 3, ".gz") == 0 ? f.substr(0, f.size() - 3) : f;
}

bool is_reference_file(const string &f)
{
    const string ext = fs::path(strip_gz(f)).extension().string();
    return ext == ".fasta" || ext == ".fa" || ext == ".fna";
}

bool list_references(const string &dir, vector<fs::path> &out)
{
    std::error_code ec;
    if (!fs::is_directory(dir, ec)) {
        cerr << "Error: reference folder not found: " << dir << endl;
        return false;
    }
    fs::directory_iterator it(dir, ec), end;
    for (; !ec && it != end; it.increment(ec)) {
        const string name = it->path().filename().string();
        if (is_reference_file(name))
            out.push_back(it->path());
        else
            cout << "Skipping " << name << " (not a reference file: .fasta, .fa or .fna, optionally .gz)"
                 << endl;
    }
    if (ec) {
        cerr << "Error: cannot list the reference folder " << dir << ": " << ec.message() << endl;
        return false;
    }
    if (out.empty()) {
        cerr << "Error: no reference files (.fasta, .fa or .fna, optionally .gz) in " << dir << endl;
        return false;
    }
    return true;
}

bool prepare_results(const string &dir)
{
    std::error_code ec;
    if (fs::is_directory(dir, ec))
        return true;
    if (fs::exists(dir, ec)) {
        cerr << "Error: results path exists and is not a folder: " << dir << endl;
        return false;
    }
    fs::create_directories(dir, ec);
    if (ec || !fs::is_directory(dir)) {
        cerr << "Error: cannot create the results folder " << dir << ": "
             << (ec ? ec.message() : "not a folder") << endl;
        return false;
    }
    return true;
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
         << "  --gpu            Scan on the GPU (the only path of this build)\n"
         << "  --device=N       CUDA device ordinal (default 0)\n"
         << "  --cpu, --probe=batched\n"
         << "                   The reference's CPU paths: not in this build; the scan runs\n"
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
    auto &o = KmerDatabase::gpuOptions();
    auto intOpt = [](const string &arg, size_t n, int &out, int lo = 1) {
        if (parse_int(arg.substr(n), lo, out))
            return true;
        cerr << "Invalid value for option: " << arg << " (expected an integer >= " << lo << ")" << endl;
        return false;
    };
    for (int a = first; a < argc; a++) {
        const string arg = argv[a];
        if (arg == "--gpu")
            o.enable = 1;
        else if (arg == "--cpu" || arg == "--probe=batched") {
            o.enable = 0;
            cerr << "Warning: " << arg << " selects the reference's CPU path, which this build does "
                 << "not have; scanning on the GPU (identical rows)" << endl;
        } else if (arg == "--sync")
            o.sync = true;
        else if (arg.rfind("--batch-mb=", 0) == 0) {
            if (!intOpt(arg, 11, o.batchMB))
                return false;
        } else if (arg.rfind("--streams=", 0) == 0) {
            if (!intOpt(arg, 10, o.streams))
                return false;
        } else if (arg == "--gpus=all")
            o.gpus = 0;
        else if (arg == "--gpus=0") {
            cerr << "Invalid value for option: --gpus=0 (use --gpus=all for every device, --cpu for none)"
                 << endl;
            return false;
        } else if (arg.rfind("--gpus=", 0) == 0) {
            if (!intOpt(arg, 7, o.gpus))
                return false;
        } else if (arg.rfind("--device=", 0) == 0) {
            if (!intOpt(arg, 9, o.device, 0))
                return false;
        } else if (arg == "--no-peer")
            o.noPeer = true;
        else if (arg.rfind("--db=", 0) == 0 && arg.size() > 5)
            panel.dbs.push_back(arg.substr(5));
        else if (arg.rfind("--db-list=", 0) == 0 && arg.size() > 10)
            panel.listFile = arg.substr(10);
        else if (arg.rfind("--resident=", 0) == 0) {
            if (!intOpt(arg, 11, panel.resident, 0))
                return false;
        } else if (arg == "--sort-queries")
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
                cerr << "Invalid value for option: " << arg << " (expected 0.1 .. 0.95)" << endl;
                return false;
            }
            o.hashLoadFactor = v;
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
