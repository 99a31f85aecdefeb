// Command-line helpers shared by the fastibs, fastibsmapper and KDBIntersect
// tools, with the reference's messages (src/CliInput.hpp:108-235): a KMC
// dataset folder resolved to "<folder>/<prefix>", the reference files of a
// folder, the results folder, the per-reference error log.
#pragma once

#include <filesystem>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

namespace ibs_cli {

namespace fs = std::filesystem;
using std::cerr;
using std::cout;
using std::endl;
using std::string;
using std::vector;

inline void trim_slash(string &p)
{
    if (!p.empty() && p.back() == '/')
        p.pop_back();
}

// The KMC prefix in a dataset folder: the name before ".kmc_" of the first
// such file; "" when there is none or the folder cannot be listed.
inline string find_prefix(const string &dir)
{
    std::error_code ec;
    for (fs::directory_iterator it(dir, ec), end; !ec && it != end; it.increment(ec)) {
        const string f = it->path().filename().string();
        const size_t pos = f.find(".kmc_");
        if (pos != string::npos)
            return f.substr(0, pos);
    }
    return "";
}

// A KMC dataset folder -> "<dir>/<prefix>"; false after one error line when
// the folder is missing or holds no <prefix>.kmc_pre + .kmc_suf pair.
inline bool resolve_database(const string &dir, string &prefixPath)
{
    std::error_code ec;
    if (!fs::is_directory(dir, ec)) {
        cerr << "Error: KMC database folder not found: " << dir;
        if (fs::exists(dir + ".kmc_pre", ec))
            cerr << " (this is a KMC prefix; pass the folder that holds "
                 << fs::path(dir).filename().string() << ".kmc_pre / .kmc_suf)";
        cerr << endl;
        return false;
    }
    const string prefix = find_prefix(dir);
    const string path = dir + "/" + prefix;
    if (prefix.empty() || !fs::exists(path + ".kmc_pre", ec) || !fs::exists(path + ".kmc_suf", ec)) {
        cerr << "Error: no KMC database (<prefix>.kmc_pre and <prefix>.kmc_suf) in " << dir << endl;
        return false;
    }
    prefixPath = path;
    return true;
}

inline string strip_gz(const string &f)
{
    return f.size() > 3 && f.compare(f.size() - 3, 3, ".gz") == 0 ? f.substr(0, f.size() - 3) : f;
}

inline bool is_reference_file(const string &f)
{
    const string ext = fs::path(strip_gz(f)).extension().string();
    return ext == ".fasta" || ext == ".fa" || ext == ".fna";
}

inline bool list_references(const string &dir, vector<fs::path> &out)
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

inline bool prepare_results(const string &dir)
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

inline void log_reference_error(const string &refName, const std::exception &e)
{
    cerr << "Error processing reference " << refName << ": " << e.what() << " (also in log.txt)"
         << endl;
    std::ofstream log("log.txt", std::ios::app);
    if (log.is_open())
        log << "Error processing reference: " << refName << endl << e.what() << endl;
    else
        cout << "Unable to open log file." << endl;
}

} // namespace ibs_cli
