// gpu_contractor.hpp -- the reference-facing C++ interface of the B200 path.
//
// Mirrors, over the C ABI of include/cuttlefish_gpu.h, the two interfaces the
// reference plugs its compaction into:
//   * the T_App<k> concept that Application<MAX_K, T_App> instantiates
//     (explicit T_App(const Build_Params&); void construct(); src/Application.cpp:9-57,
//     include/Read_CdBG.hpp:72,85) -- GPU_Contractor<k> below, a drop-in for
//     dBG_Contractor<k> (src/dBG_Contractor.cpp:19-112);
//   * the Subgraphs_Manager<k, false> surface (include/Subgraphs_Manager.hpp:80-134):
//     graph_count(), graph_ID(h), finalize(), process(), trivial_mtig_count(),
//     icc_count(), estimate_size_max(), RSS().  add_super_kmer(...) is replaced by
//     partition(), which takes the whole packed input: per-super-k-mer host calls
//     cannot feed a GPU, so Graph_Partitioner::partition is fused into the device run.
#pragma once

#include "cuttlefish_gpu.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace cuttlefish_b200 {

// The subset of Build_Params (include/Build_Params.hpp) the compaction path reads.
struct Build_Params {
    bool is_read_graph = false, is_ref_graph = true;
    std::vector<std::string> seq_paths;     // -s / -l / -d, resolved
    uint16_t k = 27;                        // -k
    uint32_t cutoff = 0;                    // -c (0: 1 for --ref, 2 for --read)
    uint16_t min_len = 20;                  // --min-len
    uint16_t thread_count = 0;              // -t (host threads for input parsing)
    std::string output_prefix;              // -o; the unitigs go to <prefix>.fa
    std::string working_dir = ".";          // -w
    int device = 0;                         // GPU ordinal
    uint32_t table_load_pct = 0;            // subgraph-table sizing hint (see cfg_params)
    uint32_t effective_cutoff() const { return cutoff ? cutoff : (is_read_graph ? 2u : 1u); }
    std::string output_file_path() const { return output_prefix + ".fa"; }   // include/Build_Params.hpp:150
};

class cfg_error : public std::runtime_error {
public:
    cfg_error(const std::string& what, int code) : std::runtime_error(what), code(code) {}
    int code;
};

// Subgraphs_Manager<k,false>-shaped owner of one GPU context.
class Subgraphs_Manager {
public:
    Subgraphs_Manager(uint16_t k, uint16_t l, uint32_t cutoff, int device, uint32_t table_load_pct = 0) {
        cfg_params p{};
        p.k = k; p.l = l; p.cutoff = cutoff; p.graph_count = 16384; p.table_load_pct = table_load_pct;
        check(cfg_create(device, &p, &ctx_), "cfg_create");
    }
    ~Subgraphs_Manager() { cfg_destroy(ctx_); }
    Subgraphs_Manager(const Subgraphs_Manager&) = delete;
    Subgraphs_Manager& operator=(const Subgraphs_Manager&) = delete;

    static constexpr uint64_t graph_count() { return 16384; }                 // include/Atlas.hpp:33-35
    static uint64_t graph_ID(uint64_t h) { return h & (graph_count() - 1); }  // include/Subgraphs_Manager.hpp:130

    // Graph_Partitioner::partition + every add_super_kmer call, for one packed input.
    void partition(const cfg_packed& in) {
        check(cfg_submit_packed(ctx_, in.words, in.n_bases, in.frag_off, in.frag_len, in.n_frags), "cfg_submit_packed");
    }
    // The same from FASTA / FASTQ text, parsed on the device.
    void partition_text(const char* text, uint64_t bytes) { check(cfg_submit_text(ctx_, text, bytes), "cfg_submit_text"); }
    void finalize() {}   // the device buckets need no flush
    // Subgraphs_Manager::process: build and contract every subgraph.
    void process() {
        check(cfg_run(ctx_), "cfg_run");
        check(cfg_fetch_counts(ctx_, &res_.counts), "cfg_fetch_counts");
    }
    // The outputs of process() in host memory (trivial unitigs, lm-tigs).
    const cfg_results& fetch() {
        check(cfg_fetch(ctx_, &res_), "cfg_fetch");
        return res_;
    }
    uint64_t trivial_mtig_count() const { return res_.counts.n_trivial; }
    uint64_t icc_count() const { return res_.counts.n_icc; }
    uint64_t estimate_size_max() const { return 0; }                          // the reference returns 0 too
    std::size_t RSS() const { return 0; }                                    // tables live on the device
    const cfg_results& results() const { return res_; }
    cfg_ctx* context() const { return ctx_; }

private:
    void check(int rc, const char* what) {
        if (rc != CFG_OK)
            throw cfg_error(std::string(what) + ": " + (ctx_ ? std::string(cfg_last_error_string(ctx_))
                                                             : "error code " + std::to_string(rc)), rc);
    }
    cfg_ctx* ctx_ = nullptr;
    cfg_results res_{};
};

// Reads the records of the inputs (FASTA or FASTQ, plain or gzip) into one
// concatenation with offsets, files in decreasing size as Graph_Partitioner
// orders its sources (src/Graph_Partitioner.cpp:121-128).
struct Records {
    std::string seq;
    std::vector<uint64_t> off{0};
};
Records read_records(const std::vector<std::string>& paths);

// Joins lm-tigs into maximal unitigs and writes <prefix>.fa; returns unitig count.
uint64_t write_unitigs(const std::string& path, uint32_t k, const cfg_results& r);

// The inputs' text joined into one FASTA or one FASTQ text (files largest first,
// each ending in a newline); empty when the files mix the two formats.
std::string read_text(const std::vector<std::string>& paths, bool& mixed);

// T_App<k>: drop-in for dBG_Contractor<k> in Application<MAX_K, T_App>.
template <uint16_t k>
class GPU_Contractor {
public:
    explicit GPU_Contractor(const Build_Params& p) : p_(p) {
        if (p.k != k) throw cfg_error("GPU_Contractor<k> instantiated for another k", CFG_ERR_BAD_INPUT);
    }
    void construct();   // defined in gpu_contractor.cpp for the runtime k

private:
    Build_Params p_;
};

// Runtime-k body of GPU_Contractor<k>::construct (dBG_Contractor::construct,
// src/dBG_Contractor.cpp:30-112): read, partition, process, collate, write.
void construct_gpu(const Build_Params& p);

template <uint16_t k>
inline void GPU_Contractor<k>::construct() { construct_gpu(p_); }

}  // namespace cuttlefish_b200
