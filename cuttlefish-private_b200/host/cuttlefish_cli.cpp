// cuttlefish_cli.cpp -- `cuttlefish build` with the reference's options
// (src/main.cpp:29-59, src/commands.cpp:30-198) over the B200 path.
#include "gpu_contractor.hpp"

#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

namespace {

using cuttlefish_b200::Build_Params;

void usage() {
    std::cout << "cuttlefish build: construct the compacted de Bruijn graph on a B200 GPU\n"
                 "  -s, --seq FILE[,FILE..]   input files (FASTA / FASTQ, optionally gzipped)\n"
                 "  -l, --list FILE           files listing inputs, one per line\n"
                 "  -d, --dir DIR             directories of inputs\n"
                 "  -k, --kmer-len K          k-mer length (odd, <= 127; default 27)\n"
                 "  -c, --cutoff C            (k+1)-mer frequency cutoff (default: refs 1, reads 2)\n"
                 "      --read | --ref        read or reference de Bruijn graph\n"
                 "      --min-len L           minimizer length (default 20)\n"
                 "  -o, --output PREFIX       output; unitigs go to PREFIX.fa\n"
                 "  -w, --work-dir DIR        working directory (default .)\n"
                 "  -t, --threads N           accepted (host parsing is single pass)\n"
                 "      --gpu N               device ordinal (default 0)\n"
                 "      --subgraph-count N, --vertex-part-count N, --lmtig-bucket-count N, --gmtig-bucket-count N,\n"
                 "      -m, --max-memory GB, --unrestrict-memory, --idx   accepted and ignored, as in the reference\n";
}

std::vector<std::string> split_commas(const std::string& v) {
    std::vector<std::string> out;
    std::stringstream ss(v);
    std::string item;
    while (std::getline(ss, item, ',')) if (!item.empty()) out.push_back(item);
    return out;
}

int cf_build(int argc, char** argv) {
    Build_Params p;
    bool read = false, ref = false;
    std::vector<std::string> seqs, lists, dirs;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto val = [&](void) -> std::string {
            if (i + 1 >= argc) throw std::runtime_error("missing value for " + a);
            return argv[++i];
        };
        if (a == "-h" || a == "--help") { usage(); return 0; }
        else if (a == "-s" || a == "--seq") for (auto& x : split_commas(val())) seqs.push_back(x);
        else if (a == "-l" || a == "--list") for (auto& x : split_commas(val())) lists.push_back(x);
        else if (a == "-d" || a == "--dir") for (auto& x : split_commas(val())) dirs.push_back(x);
        else if (a == "-k" || a == "--kmer-len") p.k = (uint16_t)std::stoi(val());
        else if (a == "-c" || a == "--cutoff") p.cutoff = (uint32_t)std::stoul(val());
        else if (a == "--min-len") p.min_len = (uint16_t)std::stoi(val());
        else if (a == "-o" || a == "--output") p.output_prefix = val();
        else if (a == "-w" || a == "--work-dir") p.working_dir = val();
        else if (a == "-t" || a == "--threads") p.thread_count = (uint16_t)std::stoi(val());
        else if (a == "--gpu") p.device = std::stoi(val());
        else if (a == "--table-load-pct") p.table_load_pct = (uint32_t)std::stoul(val());
        else if (a == "--read") read = true;
        else if (a == "--ref") ref = true;
        else if (a == "--subgraph-count" || a == "--vertex-part-count" || a == "--lmtig-bucket-count" ||
                 a == "--gmtig-bucket-count" || a == "-m" || a == "--max-memory") val();
        else if (a == "--unrestrict-memory" || a == "--idx") {}
        else if (a == "--color" || a == "--path-cover" || a == "-f" || a == "--format")
            throw std::runtime_error(a + " is not supported by the GPU path");
        else throw std::runtime_error("unknown option " + a);
    }
    for (const auto& l : lists) {
        std::ifstream in(l);
        if (!in) throw std::runtime_error("cannot open list " + l);
        std::string line;
        while (std::getline(in, line)) if (!line.empty()) seqs.push_back(line);
    }
    for (const auto& d : dirs)
        for (const auto& e : std::filesystem::directory_iterator(d))
            if (e.is_regular_file()) seqs.push_back(e.path().string());
    // Build_Params::is_valid (src/Build_Params.cpp:97-218)
    bool valid = true;
    if (seqs.empty()) { std::cout << "No sequence input provided for compacted de Bruijn graph construction.\n"; valid = false; }
    if ((p.k % 2) == 0 || p.k == 1 || p.k > 127) { std::cout << "The k-mer length (k) needs to be odd and within 127.\n"; valid = false; }
    if (read && ref) { std::cout << "Both read and reference de Bruijn graph specified.\n"; valid = false; }
    if (p.output_prefix.empty()) { std::cout << "An output path (-o) is required.\n"; valid = false; }
    if (p.min_len == 0 || p.min_len > 32 || p.min_len + 1 > p.k) { std::cout << "The minimizer length must be within [1, min(k-1, 32)].\n"; valid = false; }
    if (!valid) { std::cout << "Invalid input configuration. Aborting.\n"; return 1; }
    p.is_read_graph = read;
    p.is_ref_graph = !read;
    if (p.is_ref_graph && p.effective_cutoff() != 1) std::cout << "WARNING: cutoff frequency specified not to be 1 on reference sequences.\n";
    p.seq_paths = seqs;
    cuttlefish_b200::construct_gpu(p);
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2 || std::string(argv[1]) != "build") {
        std::cout << "usage: cuttlefish build [options]   (cuttlefish build --help)\n";
        return argc < 2 ? 1 : (std::string(argv[1]) == "-h" || std::string(argv[1]) == "--help" ? 0 : 1);
    }
    try {
        return cf_build(argc - 1, argv + 1);
    } catch (const std::exception& e) {
        std::cerr << "Error: " << e.what() << "\n";
        return 1;
    }
}
