// The reference's own discontinuity-graph phases -- Discontinuity_Graph_Contractor,
// Contracted_Graph_Expander, Unitig_Collator, compiled from its sources where they lie
// -- run on what the B200 path's GPU_Subgraphs_Manager leaves in the reference's
// Discontinuity_Graph and output buffers, in the order dBG_Contractor<k>::construct<false>
// runs them (src/dBG_Contractor.cpp:30-112, which this driver follows step by step with
// the GPU manager in place of Subgraphs_Manager + Graph_Partitioner).  The reference
// writes <output>.fa.  Test infrastructure: built by tests/dropin/Makefile (k = FIXED_K).
//
//     sgm_dropin <read|ref> <output prefix> <working dir> <input file>...
#include "Build_Params.hpp"
#include "Contracted_Graph_Expander.hpp"
#include "Data_Logistics.hpp"
#include "Discontinuity_Graph.hpp"
#include "Discontinuity_Graph_Contractor.hpp"
#include "Output_Sink.hpp"
#include "State_Config.hpp"
#include "Unitig_Collator.hpp"
#include "dBG_Contractor.hpp"
#include "parlay/parallel.h"
#include "reference_subgraphs.hpp"

#include <exception>
#include <iostream>
#include <optional>
#include <string>
#include <vector>

constexpr uint16_t K = FIXED_K;
typedef cuttlefish::dBG_Contractor<K> Contractor;   // only its typedefs are used

int main(int argc, char** argv) {
    if (argc < 5) {
        std::cerr << "usage: sgm_dropin <read|ref> <output prefix> <working dir> <input file>...\n";
        return 2;
    }
    const bool read = std::string(argv[1]) == "read";
    const std::vector<std::string> seqs(argv + 4, argv + argc);
    namespace def = cuttlefish::_default;
    const Build_Params params(read, !read, seqs, std::nullopt, std::nullopt, K, std::nullopt, false,
                              def::SUBGRAPH_COUNT, def::VERTEX_PART_COUNT, def::LMTIG_BUCKET_COUNT,
                              def::GMTIG_BUCKET_COUNT, "", "", 1, std::nullopt, false, false, def::MIN_LEN,
                              argv[2], cuttlefish::Output_Format::fa, false, false, argv[3], false, false, false,
                              false);
    try {
        cuttlefish::Edge_Frequency::set_edge_threshold(params.cutoff());
        const Data_Logistics logistics(params);
        Output_Sink<Contractor::sink_t> output_sink;
        Contractor::op_buf_list_t op_buf(parlay::num_workers(), Contractor::op_buf_t(output_sink.sink()));
        const auto op_file_path = logistics.output_file_path();
        clear_file(op_file_path);
        output_sink.init_sink(op_file_path);

        cuttlefish::Discontinuity_Graph<K, false> gamma(params, logistics);
        {
            cuttlefish_b200::GPU_Subgraphs_Manager<K> G(logistics, params.min_len(), gamma, op_buf);
            bool mixed = false;
            const std::string text = cuttlefish_b200::read_text(params.sequence_input().seqs(), mixed);
            if (mixed) throw std::runtime_error("inputs mix FASTA and FASTQ");
            G.partition_text(text.data(), text.size());
            G.finalize();
            G.process();
            std::cerr << "Trivial maximal unitig count: " << G.trivial_mtig_count() << ".\n";
        }

        Contractor::P_v_t P_v;   // path-info of vertices, one bucket per vertex partition (+ the phi partition 0)
        P_v.reserve(params.vertex_part_count() + 1);
        P_v.emplace_back();
        for (std::size_t j = 1; j <= params.vertex_part_count(); ++j)
            P_v.emplace_back(Contractor::p_v_bucket_t(logistics.vertex_path_info_buckets_path() + "_" + std::to_string(j),
                                                      128 * 1024));
        {
            cuttlefish::Discontinuity_Graph_Contractor<K, false> contractor(gamma, P_v, logistics);
            contractor.contract();
            gamma.close();
        }
        Contractor::P_e_t P_e;   // path-info of edges, one bucket per lm-tig bucket (+ partition 0)
        P_e.reserve(params.lmtig_bucket_count() + 1);
        P_e.emplace_back();
        for (std::size_t b = 1; b <= params.lmtig_bucket_count(); ++b)
            P_e.emplace_back(Contractor::p_e_bucket_t(logistics.edge_path_info_buckets_path() + "_" + std::to_string(b),
                                                      128 * 1024));
        {
            cuttlefish::Contracted_Graph_Expander<K, false> expander(gamma, P_v, P_e, logistics);
            expander.expand();
        }
        force_free(P_v);
        {
            cuttlefish::Unitig_Collator<K, false> collator(gamma, P_e, logistics, op_buf, params.gmtig_bucket_count());
            collator.collate();
        }
        for (auto& b : op_buf) b.unwrap().close();
        output_sink.close_sink();
    } catch (const cuttlefish_b200::cfg_error& e) {
        std::cerr << "GPU_Subgraphs_Manager<" << K << ">: " << e.what() << "\n";
        return 3;
    }
    return 0;
}
