// gpu_contractor.cpp -- input reading and the construct() phases of the B200 path
// (the CLI is cuttlefish_cli.cpp).
#include "gpu_contractor.hpp"

#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>

namespace cuttlefish_b200 {

namespace {

double since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// One whole (possibly gzipped) file in memory.
std::string slurp(const std::string& path) {
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f) throw cfg_error("cannot open input " + path, CFG_ERR_BAD_INPUT);
    gzbuffer(f, 1 << 20);
    std::string out;
    std::vector<char> buf(1 << 22);
    for (;;) {
        const int n = gzread(f, buf.data(), (unsigned)buf.size());
        if (n < 0) { gzclose(f); throw cfg_error("cannot read input " + path, CFG_ERR_BAD_INPUT); }
        if (n == 0) break;
        out.append(buf.data(), (size_t)n);
    }
    gzclose(f);
    return out;
}

// FASTA: a record's sequence is its lines joined (RabbitFX chunkListFormat,
// include/RabbitFX/io/Formater.cpp:87-130); FASTQ: the second line of each record.
void parse_into(const std::string& text, Records& r) {
    size_t i = 0;
    const size_t n = text.size();
    while (i < n && (text[i] == '\n' || text[i] == '\r')) ++i;
    if (i == n) return;
    if (text[i] == '@') {
        while (i < n) {
            size_t e = text.find('\n', i);             // header
            if (e == std::string::npos) break;
            size_t s = e + 1, t = text.find('\n', s);   // sequence
            if (t == std::string::npos) t = n;
            r.seq.append(text, s, t - s);
            r.off.push_back(r.seq.size());
            size_t p = t + 1;                            // '+' line, then quality
            for (int skip = 0; skip < 2 && p < n; ++skip) {
                const size_t q = text.find('\n', p);
                p = q == std::string::npos ? n : q + 1;
            }
            i = p;
            while (i < n && (text[i] == '\n' || text[i] == '\r')) ++i;
        }
        return;
    }
    bool in_rec = false;
    while (i < n) {
        size_t e = text.find('\n', i);
        if (e == std::string::npos) e = n;
        if (text[i] == '>') {
            if (in_rec) r.off.push_back(r.seq.size());
            in_rec = true;
        } else if (in_rec) {
            r.seq.append(text, i, e - i);
        }
        i = e + 1;
    }
    if (in_rec) r.off.push_back(r.seq.size());
}

}  // namespace

Records read_records(const std::vector<std::string>& paths) {
    std::vector<std::pair<uint64_t, std::string>> by_size;
    for (const auto& p : paths) {
        std::error_code ec;
        const auto sz = std::filesystem::file_size(p, ec);
        if (ec) throw cfg_error("cannot open input " + p, CFG_ERR_BAD_INPUT);
        by_size.emplace_back(sz, p);
    }
    std::stable_sort(by_size.begin(), by_size.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    Records r;
    for (const auto& e : by_size) parse_into(slurp(e.second), r);
    return r;
}

std::string read_text(const std::vector<std::string>& paths, bool& mixed) {
    std::vector<std::pair<uint64_t, std::string>> by_size;
    for (const auto& p : paths) {
        std::error_code ec;
        const auto sz = std::filesystem::file_size(p, ec);
        if (ec) throw cfg_error("cannot open input " + p, CFG_ERR_BAD_INPUT);
        by_size.emplace_back(sz, p);
    }
    std::stable_sort(by_size.begin(), by_size.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    std::string all;
    int fmt = -1;   // 1 FASTQ, 0 FASTA
    mixed = false;
    for (const auto& e : by_size) {
        std::string t = slurp(e.second);
        size_t i = 0;
        while (i < t.size() && (t[i] == '\n' || t[i] == '\r')) ++i;
        if (i == t.size()) continue;
        const int f = t[i] == '@';
        if (fmt >= 0 && f != fmt) { mixed = true; return std::string(); }
        fmt = f;
        all += t;
        if (all.back() != '\n') all += '\n';
    }
    return all;
}

uint64_t write_unitigs(const std::string& path, uint32_t k, const cfg_results& r) {
    char* stitched = nullptr;
    uint64_t bytes = 0, n_units = 0, n_cycles = 0;
    const int rc = cfg_collate_lmtigs(k, r.lmtigs, r.counts.n_lmtig, r.lmtig_text, &stitched, &bytes, &n_units, &n_cycles);
    if (rc != CFG_OK) throw cfg_error("cfg_collate_lmtigs failed", rc);
    std::ofstream out(path, std::ios::binary);
    if (!out) { cfg_free(stitched); throw cfg_error("cannot write " + path, CFG_ERR_BAD_INPUT); }
    out.write(r.fasta, (std::streamsize)r.counts.fasta_bytes);
    out.write(stitched, (std::streamsize)bytes);
    cfg_free(stitched);
    if (!out) throw cfg_error("error writing " + path, CFG_ERR_BAD_INPUT);
    return r.counts.n_trivial + n_units;
}

void construct_gpu(const Build_Params& p) {
    const auto t0 = std::chrono::steady_clock::now();
    bool mixed = false;
    std::string text = read_text(p.seq_paths, mixed);
    Subgraphs_Manager G(p.k, p.min_len, p.effective_cutoff(), p.device,
                        p.table_load_pct ? p.table_load_pct : (p.is_read_graph ? 15u : 0u));
    cfg_packed packed{};
    if (!mixed) {
        // parsed on the device (records, line joins, fragments)
        G.partition_text(text.data(), text.size());
        std::cerr << "Read " << text.size() << " bytes of " << p.seq_paths.size()
                  << " input file(s); parsed on the device. Time taken: " << since(t0) << " seconds.\n";
    } else {
        Records recs = read_records(p.seq_paths);
        int rc = cfg_pack_records(recs.seq.data(), recs.off.data(), recs.off.size() - 1, p.k, 1, &packed);
        if (rc != CFG_OK) throw cfg_error("cfg_pack_records failed", rc);
        std::cerr << "Read " << recs.off.size() - 1 << " records, " << packed.n_bases << " bases in fragments. Time taken: "
                  << since(t0) << " seconds.\n";
        G.partition(packed);
    }
    std::string().swap(text);
    const auto t1 = std::chrono::steady_clock::now();
    G.finalize();
    G.process();
    float ms[4] = {0, 0, 0, 0};
    cfg_last_timings(G.context(), ms);
    std::cerr << "Sequence splitting into subgraphs completed. Time taken: " << (ms[0] + ms[1]) / 1e3 << " seconds.\n";
    std::cerr << "Subgraphs construction and contraction completed. Time taken: " << ms[2] / 1e3 << " seconds.\n";
    std::cerr << "Trivial maximal unitig count: " << G.trivial_mtig_count() << ".\n";
    std::cerr << "Isolated cycle count: " << G.icc_count() << ".\n";
    std::cerr << "lm-tig count: " << G.results().counts.n_lmtig << ".\n";
    if (packed.words) cfg_packed_free(&packed);
    const auto t2 = std::chrono::steady_clock::now();
    // the discontinuity-graph phases, on the device
    const char* fa = nullptr;
    uint64_t bytes = 0, units = 0;
    float ums = 0;
    const int rc = cfg_unitigs(G.context(), &fa, &bytes, &units, &ums);
    if (rc != CFG_OK) throw cfg_error(std::string("cfg_unitigs: ") + cfg_last_error_string(G.context()), rc);
    std::ofstream out(p.output_file_path(), std::ios::binary);
    if (!out) throw cfg_error("cannot write " + p.output_file_path(), CFG_ERR_BAD_INPUT);
    out.write(fa, (std::streamsize)bytes);
    if (!out) throw cfg_error("error writing " + p.output_file_path(), CFG_ERR_BAD_INPUT);
    std::cerr << "Collated " << units << " maximal unitigs into " << p.output_file_path() << ". Time taken: "
              << since(t2) << " seconds (device " << ums / 1e3 << ").\n";
    std::cerr << "Device phases and transfers: " << std::chrono::duration<double>(t2 - t1).count()
              << " seconds; total: " << since(t0) << " seconds.\n";
}

}  // namespace cuttlefish_b200
