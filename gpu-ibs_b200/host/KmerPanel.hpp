// KmerPanel: N sample databases scanned against a reference in one pass
// (the reference's panel mode, src/KmerPanel.hpp): the reference is read and
// packed once and uploaded once, the databases are taken in rounds of up to
// 16 that fit the device (or --resident=N), and each round is ONE joint
// table (ibs_panel_table: every key once, with a mask of the samples that
// hold it) scanned in one pass: one bucket load per position serves the
// whole round. Every database's TSV is the file a single run writes (the
// same Window records through the same writer). A single round stays
// resident for the next reference, as the reference does
// (src/KmerPanel.hpp:122-135, :213-222).
#pragma once

#include <algorithm>
#include <chrono>
#include <iostream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "KmerDatabase.hpp"

class KmerPanel
{
public:
    // prefixes[i]: database i's KMC path prefix; names[i]: its output name
    // (the folder's name); resident: at most this many per round (0: as many
    // as fit). Throws on a k mismatch or k > 32 (src/KmerPanel.hpp:30-54).
    KmerPanel(const std::vector<std::string> &prefixes, const std::vector<std::string> &names,
              int resident)
        : residentCap(resident)
    {
        if (prefixes.empty() || prefixes.size() != names.size())
            throw std::runtime_error("KmerPanel: no databases");
        for (size_t i = 0; i < prefixes.size(); i++) {
            Member m;
            m.prefix = prefixes[i];
            m.name = names[i];
            m.db = std::make_unique<KmerDatabase>(prefixes[i]);
            if (!members.empty() && m.db->getKmerSize() != members[0].db->getKmerSize())
                throw std::runtime_error("KmerPanel: " + m.name + " has k=" +
                                         std::to_string(m.db->getKmerSize()) + " but " +
                                         members[0].name + " has k=" +
                                         std::to_string(members[0].db->getKmerSize()) +
                                         "; a panel shares one k");
            // joint tables hold 64-bit codes; fastibs scans a k > 32 panel
            // as single runs instead, as the reference does
            if (m.db->getKmerSize() > 32)
                throw std::runtime_error("KmerPanel: k=" + std::to_string(m.db->getKmerSize()) +
                                         " > 32 has no panel path");
            members.push_back(std::move(m));
        }
    }

    size_t size() const { return members.size(); }
    const std::string &name(size_t i) const { return members[i].name; }
    unsigned kmerSize() const { return members[0].db->getKmerSize(); }
    KmerDatabase &database(size_t i) { return *members[i].db; }

    // One reference against every member whose outPaths[i] is non-empty.
    void processReference(const std::string &refPath, const std::vector<std::string> &outPaths,
                          int windowSize)
    {
        if (outPaths.size() != members.size())
            throw std::runtime_error("KmerPanel: one output path per database expected");
        std::vector<size_t> active;
        for (size_t i = 0; i < members.size(); i++)
            if (!outPaths[i].empty())
                active.push_back(i);
        if (active.empty())
            return;
        const auto tRef = std::chrono::steady_clock::now();
        auto since = [](const std::chrono::steady_clock::time_point &t) {
            return std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
        };
        const unsigned k = kmerSize();
        std::cout << "Window size: " << windowSize << std::endl;
        std::cout << "Kmer size: " << k << std::endl;
        std::cout << "K-mer path: fused GPU encode+probe (sm_100a), " << active.size()
                  << " databases per reference pass" << std::endl;
        KmerDatabase::checkWindow(windowSize, k);

        KmerDatabase::PackedReference ref;
        ibs_reference *dref = KmerDatabase::loadReference(refPath, ref);
        std::unique_ptr<ibs_reference, void (*)(ibs_reference *)> refGuard(dref, ibs_reference_free);
        const uint64_t nWin = ibs_window_count(ref.lens.data(), (uint32_t)ref.lens.size(),
                                               (uint32_t)windowSize, k);
        std::cout << "Number of chunks: " << nWin << std::endl;

        std::vector<std::vector<size_t>> rounds;
        if (!keptResident.empty() && keptResident == active)
            rounds = {active};
        else {
            releaseAll();
            rounds = planRounds(active);
        }
        std::cout << "[panel] " << active.size() << " databases in " << rounds.size()
                  << (rounds.size() == 1 ? " round" : " rounds") << std::endl;

        double setupTotal = 0, statsTotal = 0, writeTotal = 0;
        std::string writeErrors;
        for (size_t r = 0; r < rounds.size(); r++) {
            const std::vector<size_t> &round = rounds[r];
            auto t0 = std::chrono::steady_clock::now();
            if (!joint)
                buildJoint(round);
            const double setupSec = since(t0);
            setupTotal += setupSec;

            t0 = std::chrono::steady_clock::now();
            std::cout << "Calculating stats" << std::endl;
            std::vector<ibs_window> rows(std::max<uint64_t>(1, nWin * round.size()));
            KmerDatabase::check(ibs_panel_table_scan(joint, dref, (uint32_t)windowSize, rows.data(),
                                                     nWin * round.size()),
                                "ibs_panel_table_scan");
            const double statsSec = since(t0);
            statsTotal += statsSec;

            t0 = std::chrono::steady_clock::now();
            std::cout << "Writing stats to file" << std::endl;
            for (size_t j = 0; j < round.size(); j++) {
                try {
                    KmerDatabase::writeStats(outPaths[round[j]],
                                             KmerDatabase::toWindows(ref, rows.data() + j * nWin,
                                                                     windowSize, k));
                } catch (const std::exception &e) {
                    writeErrors += (writeErrors.empty() ? "" : "; ") + std::string(e.what());
                }
            }
            const double writeSec = since(t0);
            writeTotal += writeSec;
            if (rounds.size() > 1)
                releaseAll();
            std::cout << "[panel] round " << r + 1 << "/" << rounds.size() << ": " << round.size()
                      << " databases, setup " << setupSec << " s, stats " << statsSec
                      << " s, write " << writeSec << " s" << std::endl;
        }
        keptResident = rounds.size() == 1 ? rounds[0] : std::vector<size_t>{};
        std::cout << "Scan phases: setup " << setupTotal << " s, read " << ref.readSec
                  << " s, window " << ref.packSec << " s, stats " << statsTotal << " s, write "
                  << writeTotal << " s" << std::endl;
        const double total = since(tRef);
        std::cout << "[panel] reference done: " << active.size() << " databases in "
                  << rounds.size() << (rounds.size() == 1 ? " round, " : " rounds, ") << total
                  << " s, per database " << total / active.size() << " s" << std::endl;
        if (!writeErrors.empty())
            throw std::runtime_error(writeErrors);
    }

private:
    struct Member {
        std::string prefix, name;
        std::unique_ptr<KmerDatabase> db;
    };
    std::vector<Member> members;
    int residentCap = 0;
    std::vector<size_t> keptResident;
    ibs_panel_table *joint = nullptr; // the current round's table
    static constexpr double kKeysPerBucket = 3.0;

public:
    ~KmerPanel() { releaseAll(); }

private:
    void releaseAll()
    {
        if (joint) {
            ibs_panel_table_close(joint);
            joint = nullptr;
        }
        keptResident.clear();
    }

    // Upper bound of a member's share of a joint table: its keys at the
    // table's load in 32-byte buckets, plus the overflow stash.
    static uint64_t jointBytes(uint64_t keys) { return (uint64_t)(keys / kKeysPerBucket * 32 * 1.15); }

    // One joint table of the round's databases. Its size is planned for the
    // sum of their key counts (the union is at most that; the stash grows
    // if the planning is short).
    void buildJoint(const std::vector<size_t> &round)
    {
        uint64_t keys = 0;
        for (size_t i : round)
            keys += members[i].db->kmcInfo().totalKmers;
        ibs_table_opts o{};
        o.device = KmerDatabase::gpuOptions().device;
        o.keys_per_bucket = kKeysPerBucket;
        const auto t0 = std::chrono::steady_clock::now();
        KmerDatabase::check(ibs_panel_table_create(kmerSize(), keys, &o, &joint), "ibs_panel_table_create");
        for (size_t i : round)
            KmerDatabase::check(ibs_panel_table_add_kmc(joint, members[i].prefix.c_str()),
                                "ibs_panel_table_add_kmc");
        ibs_table_info ti{};
        uint32_t ns = 0;
        ibs_panel_table_info_get(joint, &ti, &ns);
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        char msg[200];
        snprintf(msg, sizeof msg, "[gpu] joint table of %u databases: %.3f s (%llu k-mers, %.2f GB on device %d)",
                 ns, sec, (unsigned long long)ti.n_keys, ti.device_bytes / 1e9, o.device);
        std::cout << msg << std::endl;
    }

    // Resident sets in order: the longest run of what is left whose tables
    // fit the device's free memory (less a margin), capped by --resident. A
    // database that fits nowhere forms a round of its own and its build
    // reports the shortfall (src/KmerPanel.hpp:282-363).
    std::vector<std::vector<size_t>> planRounds(const std::vector<size_t> &active) const
    {
        size_t cap = std::min<size_t>(active.size(), IBS_PANEL_MAX_SAMPLES);
        if (residentCap > 0)
            cap = std::min<size_t>(cap, (size_t)residentCap);
        uint64_t freeBytes = 0, totalBytes = 0;
        const bool known =
            ibs_device_memory(KmerDatabase::gpuOptions().device, &freeBytes, &totalBytes) == IBS_OK;
        const uint64_t margin = 2ull << 30; // build scratch, context, fragmentation
        std::vector<std::vector<size_t>> rounds;
        std::vector<size_t> cur;
        uint64_t curBytes = 0;
        for (size_t i : active) {
            const auto &info = members[i].db->kmcInfo();
            // its share of the joint table, and the build's transient decode buffer
            const uint64_t bytes = jointBytes(info.totalKmers);
            bool fits = cur.size() < cap;
            if (fits && known)
                fits = curBytes + bytes + margin + info.totalKmers * 8 <= freeBytes || cur.empty();
            if (!fits) {
                rounds.push_back(cur);
                cur.clear();
                curBytes = 0;
            }
            cur.push_back(i);
            curBytes += bytes;
        }
        if (!cur.empty())
            rounds.push_back(cur);
        return rounds;
    }
};
