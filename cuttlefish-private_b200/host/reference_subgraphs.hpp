// reference_subgraphs.hpp -- the B200 path behind the reference's Subgraphs_Manager.
//
// Compiled with the reference's include/ on the include path.  GPU_Subgraphs_Manager<k>
// has the constructor of Subgraphs_Manager<k, false> (include/Subgraphs_Manager.hpp:80):
// the data logistics, the minimizer length l, the discontinuity graph G and the
// per-worker output buffers op_buf; the same accessors (graph_count, G, graph_ID,
// finalize, process, trivial_mtig_count, icc_count, estimate_size_max, RSS); and
// process() leaves in those objects what Subgraph::contract leaves there
// (src/Subgraph.cpp:183-271, include/Subgraph.hpp:414-464):
//   - every lm-tig: G.add_edge(u, s_u, v, s_v, u_is_phi, v_is_phi, mtig), its label
//     carried by a Maximal_Unitig_Scratch<k> in finalize_weak form (the stored label is
//     rc(u_f) followed by u_b past its first k bases, include/Unitig_File.hpp:338-359);
//   - every isolated discontinuity vertex: G.inc_potential_phantom_edge();
//   - every trivial maximal unitig: its FASTA record appended to an op_buf buffer.
// add_super_kmer(...), which Graph_Partitioner calls once per super k-mer, is replaced
// by partition(...): the device partitions a whole packed input at once.  The edge
// frequency cutoff is the one dBG_Contractor set with Edge_Frequency::set_edge_threshold
// (src/dBG_Contractor.cpp:24), read back through Edge_Frequency's public interface.
#pragma once

#include "dBG_Contractor.hpp"        // the reference's: Discontinuity_Graph, op_buf types
#include "Directed_Vertex.hpp"
#include "Maximal_Unitig_Scratch.hpp"
#include "State_Config.hpp"
#include "gpu_contractor.hpp"

#include <cstdint>
#include <string>
#include <string_view>

namespace cuttlefish_b200 {

template <uint16_t k>
class GPU_Subgraphs_Manager {
public:
    typedef cuttlefish::Discontinuity_Graph<k, false> graph_t;
    typedef typename cuttlefish::dBG_Contractor<k>::op_buf_list_t op_buf_list_t;

    GPU_Subgraphs_Manager(const Data_Logistics& logistics, uint16_t l, graph_t& G, op_buf_list_t& op_buf, int device = 0)
        : G_(G), op_buf_(op_buf), mgr_(k, l, edge_threshold(), device, 0) {
        (void)logistics;   // the device holds every bucket: nothing is spilled to the working directory
    }

    uint64_t graph_count() const { return mgr_.graph_count(); }
    const graph_t& G() const { return G_; }
    uint64_t graph_ID(uint64_t h) const { return mgr_.graph_ID(h); }

    // Graph_Partitioner::partition and its add_super_kmer calls, for one packed input.
    void partition(const cfg_packed& in) { mgr_.partition(in); }
    void partition_text(const char* text, uint64_t bytes) { mgr_.partition_text(text, bytes); }
    void finalize() { mgr_.finalize(); }

    // Subgraphs_Manager::process: construct and contract every subgraph on the device,
    // then hand the results to G and op_buf.
    void process() {
        mgr_.process();
        const cfg_results& r = mgr_.fetch();
        for (uint64_t i = 0; i < r.counts.n_lmtig; ++i) add_lmtig(r.lmtigs[i], r.lmtig_text);
        for (uint64_t i = 0; i < r.counts.n_phantom; ++i) G_.inc_potential_phantom_edge();
        append_fasta(r.fasta, r.counts.fasta_bytes);
    }

    uint64_t trivial_mtig_count() const { return mgr_.trivial_mtig_count(); }
    uint64_t icc_count() const { return mgr_.icc_count(); }
    uint64_t estimate_size_max() const { return 0; }   // the reference returns 0 too
    std::size_t RSS() const { return 0; }               // the tables live on the device

    // The frequency threshold of the reference's Edge_Frequency: the number of times one
    // edge must be added before edge_at reports it (the threshold itself is private).
    static uint32_t edge_threshold() {
        cuttlefish::Edge_Frequency f;
        for (uint32_t c = 1; c <= 15; ++c) {
            f.add_edge<cuttlefish::side_t::back>(cuttlefish::base_t::A);
            if (f.edge_at(cuttlefish::side_t::back) == cuttlefish::base_t::A) return c;
        }
        return 15;
    }

private:
    // Kmer<k> of a cfg_lmtig k-mer: words from the lowest, the first base most significant.
    static Kmer<k> kmer_of(const uint64_t w[4]) {
        char s[k + 1];
        for (uint32_t i = 0; i < k; ++i) {
            const uint32_t bp = 2 * (k - 1 - i);
            s[i] = "ACGT"[(w[bp >> 6] >> (bp & 63)) & 3];
        }
        s[k] = '\0';
        return Kmer<k>(s);
    }

    void add_lmtig(const cfg_lmtig& m, const char* text) {
        const char* L = text + m.label_off;
        const uint32_t n = m.label_len;
        const bool u_phi = m.flags & 4, v_phi = m.flags & 8;
        const auto s_u = (m.flags & 1) ? cuttlefish::side_t::back : cuttlefish::side_t::front;
        const auto s_v = (m.flags & 2) ? cuttlefish::side_t::back : cuttlefish::side_t::front;
        // u_f: the label's first k-mer reverse complemented (finalize_weak turns it back);
        // u_b: the whole label, walked k-mer by k-mer from that first k-mer
        Maximal_Unitig_Scratch<k> mtig;
        mtig.mark_linear();
        const Kmer<k> first(L);
        mtig.unitig(cuttlefish::side_t::front).init(Directed_Vertex<k>(first.reverse_complement()));
        auto& u_b = mtig.unitig(cuttlefish::side_t::back);
        u_b.init(Directed_Vertex<k>(first));
        for (uint32_t i = k; i < n; ++i)
            if (!u_b.extend(Directed_Vertex<k>(Kmer<k>(L + i - k + 1)), L[i]))
                throw cfg_error("lm-tig revisits its first vertex", CFG_ERR_STATE);
        mtig.finalize_weak();
        G_.add_edge(u_phi ? graph_t::phi() : kmer_of(m.u), s_u, v_phi ? graph_t::phi() : kmer_of(m.v), s_v, u_phi, v_phi,
                    mtig);
    }

    // ">0\nSEQ\n" records, appended one at a time (the buffer flushes between records).
    void append_fasta(const char* fa, uint64_t bytes) {
        auto& buf = op_buf_[0].unwrap();
        uint64_t at = 0;
        while (at < bytes) {
            const std::string_view rest(fa + at, bytes - at);
            const size_t h = rest.find('\n');
            const size_t e = h == std::string_view::npos ? std::string_view::npos : rest.find('\n', h + 1);
            const size_t len = e == std::string_view::npos ? rest.size() : e + 1;
            buf += rest.substr(0, len);
            at += len;
        }
    }

    graph_t& G_;
    op_buf_list_t& op_buf_;
    Subgraphs_Manager mgr_;
};

}  // namespace cuttlefish_b200
