// fastibsmapper: the reference's mapping tool (src/FastIBSMapper.cpp) over
// the B200 library.
//
//   fastibsmapper <sourcePath> <referencePath> <resultsFolder> [options]
//
// For each reference file in <referencePath>: every base of every contig
// with the number of the KMC database's k-mers that cover it, written to
// <resultsFolder>/<database>_v_<stem>.txt (the stem without .gz and the
// FASTA extension) as "<id>\n<c0,c1,...>\n" per contig. Same arguments,
// folder checks, skip-if-exists rule, log.txt error log and exit status as
// the reference; its engine options are accepted (see GpuCli.hpp).
#include <chrono>
#include <filesystem>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "CliInput.hpp"
#include "GpuCli.hpp"
#include "KmerDatabase.hpp"

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

void usage(const char *argv0)
{
    cout << "\nFastIBS - Reference Mapping Tool (B200 build)\n"
         << "----------------------------------------------\n"
         << "Usage:\n"
         << "  " << argv0 << " <sourcePath> <referencePath> <resultsFolder> [options]\n\n"
         << "Arguments:\n"
         << "  <sourcePath>     Folder holding the KMC database files (<prefix>.kmc_pre / .kmc_suf)\n"
         << "  <referencePath>  Folder of reference genomes (*.fasta, *.fa, *.fna, optionally .gz)\n"
         << "  <resultsFolder>  Folder for the mapping files (created if missing)\n\n"
         << "Options: --device=N picks the CUDA device; the reference's other engine options\n"
         << "(--gpu, --batch-mb=, --streams=, --gpus=, --sync, --no-peer, --sort-queries, --probe=,\n"
         << "--pin-lut, --hash-lf=) are accepted; --cpu / --probe=batched run on the GPU.\n\n"
         << "Output: <resultsFolder>/<sourcePath folder>_v_<reference stem>.txt, per contig its id\n"
         << "and, on the next line, for every base the number of the database's k-mers that cover\n"
         << "it, comma-separated. Existing outputs are skipped; errors go to log.txt. Exit status 0\n"
         << "when every reference was processed or skipped, 1 otherwise.\n\n";
}

int run(int argc, char **argv)
{
    for (int a = 1; a < argc; a++)
        if (string(argv[a]) == "--version") {
            cout << "fastibsmapper (GPU-IBS, B200 scan) " << IBS_VERSION << ", sm_100a build" << endl;
            return 0;
        }
    for (int a = 1; a < argc; a++)
        if (string(argv[a]) == "-h" || string(argv[a]) == "--help") {
            usage(argv[0]);
            return 0;
        }
    if (argc < 4) {
        usage(argv[0]);
        return 1;
    }
    string source = argv[1], refPath = argv[2], results = argv[3];
    for (int a = 4; a < argc; a++) {
        const int g = ibs_cli::parse_gpu_flag(argv[a]);
        if (g == 0)
            cerr << "Unknown option: " << argv[a] << endl;
        if (g <= 0) {
            usage(argv[0]);
            return 1;
        }
    }
    ibs_cli::trim_slash(source);
    ibs_cli::trim_slash(refPath);
    ibs_cli::trim_slash(results);
    const string sourceDir = source;
    string prefix;
    if (!ibs_cli::resolve_database(sourceDir, prefix))
        return 1;
    vector<fs::path> refs;
    if (!ibs_cli::list_references(refPath, refs))
        return 1;
    const string database = fs::path(sourceDir).filename().string();
    cout << "****Database: " << database << endl;
    cout << "Using sourcePath: " << prefix << endl;
    cout << "Using referencePath: " << refPath << endl;
    cout << "Using resultsFolder: " << results << endl;
    const auto t0 = std::chrono::steady_clock::now();
    cout << "Loading KMC database from " << prefix << endl;
    std::unique_ptr<KmerDatabase> db;
    try {
        db = std::make_unique<KmerDatabase>(prefix);
    } catch (const std::exception &e) {
        cerr << "Error: " << e.what() << endl;
        return 1;
    }
    db->printKMCInfo();
    cout << "Database loaded in " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count()
         << " seconds" << endl;
    cout << "********************************************" << endl;
    if (!ibs_cli::prepare_results(results))
        return 1;
    int failed = 0;
    for (const auto &ref : refs) {
        // x.fasta -> x, x.fasta.gz -> x
        const string refName = fs::path(ibs_cli::strip_gz(ref.filename().string())).stem().string();
        cout << "Processing reference: " << refName << endl;
        const string out = results + "/" + database + "_v_" + refName + ".txt";
        if (fs::exists(out)) {
            cout << "File already exists, skipping..." << endl;
            continue;
        }
        try {
            db->produceMapping(ref.string(), out);
        } catch (const std::exception &e) {
            failed++;
            ibs_cli::log_reference_error(refName, e);
        }
    }
    if (failed)
        cerr << failed << " reference(s) failed; see log.txt" << endl;
    return failed ? 1 : 0;
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
