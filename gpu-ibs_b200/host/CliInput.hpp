// Command-line helpers shared by the fastibs and KDBIntersect tools, with
// the reference's messages (src/CliInput.hpp:108-150): a KMC dataset folder
// resolved to "<folder>/<prefix>", trailing slashes trimmed.
#pragma once

#include <filesystem>
#include <iostream>
#include <string>

namespace ibs_cli {

namespace fs = std::filesystem;
using std::cerr;
using std::endl;
using std::string;

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

} // namespace ibs_cli
