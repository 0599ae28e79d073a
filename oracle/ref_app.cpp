// The reference's own `cuttlefish build` path, compiled from its sources where they lie
// (oracle/ref_app.mk): Application<MAX_K, dBG_Contractor>(params).execute(), the call
// cf_build makes (src/commands.cpp:185), with Build_Params constructed as cf_build
// constructs it from the command line.  Partitioning, the subgraphs and the
// discontinuity-graph phases are all the reference's code, on PARLAY_NUM_THREADS
// threads; its stderr carries the phase times ("Sequence splitting into subgraphs
// completed", "Subgraphs construction and contraction completed",
// src/dBG_Contractor.cpp:58,69) and it writes <output>.fa.  Test and baseline
// infrastructure only: the timed CPU baseline and a cross-check of the oracle.
//
//     cuttlefish_ref_<k> <read|ref> <cutoff, 0: default> <output prefix> <working dir> <input file>...
#include "Application.cpp"   // the reference's src/

#include <iostream>
#include <optional>
#include <string>
#include <vector>

// Partition and bucket counts of the discontinuity-graph phases, set as the reference's
// --vertex-part-count / --lmtig-bucket-count / --gmtig-bucket-count options would set
// them: below the defaults (64, 1024, 1024), so that with the 16384 subgraph bucket
// files the process stays within the open-file limit here.  They change how the
// external-memory phases split their work on disk, not the unitigs.
constexpr std::size_t VERTEX_PARTS = 16, LMTIG_BUCKETS = 128, GMTIG_BUCKETS = 128;

int main(int argc, char** argv) {
    if (argc < 6) {
        std::cerr << "usage: cuttlefish_ref_" << cuttlefish::MAX_K
                  << " <read|ref> <cutoff, 0: default> <output prefix> <working dir> <input file>...\n";
        return 2;
    }
    const bool read = std::string(argv[1]) == "read";
    const long c = std::stol(argv[2]);
    const std::optional<uint32_t> cutoff = c > 0 ? std::optional<uint32_t>((uint32_t)c) : std::nullopt;
    const std::vector<std::string> seqs(argv + 5, argv + argc);
    namespace def = cuttlefish::_default;
    const Build_Params params(read, !read, seqs, std::nullopt, std::nullopt, cuttlefish::MAX_K, cutoff, false,
                              def::SUBGRAPH_COUNT, VERTEX_PARTS, LMTIG_BUCKETS, GMTIG_BUCKETS, "", "",
                              (uint16_t)parlay::num_workers(), std::nullopt, false,
                              false, def::MIN_LEN, argv[3], cuttlefish::Output_Format::fa, false, false, argv[4],
                              false, false, false, false);
    const Application<cuttlefish::MAX_K, cuttlefish::dBG_Contractor> app(params);
    app.execute();
    return 0;
}
