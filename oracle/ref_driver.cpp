/*
 * ref_driver.cpp -- pins the oracle to the reference's own code.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/ref.mk against the reference's
 * headers where they lie (Kmer.hpp, Directed_Vertex.hpp, Minimizer_Iterator.hpp,
 * Minimizer_Utility.hpp + the vendored wyhash.h, State_Config.hpp +
 * src/State_Config.cpp, Unitig_Scratch.hpp, Maximal_Unitig_Scratch.hpp,
 * FASTA_Record.hpp, Character_Buffer.hpp) into oracle/_ref/ref_driver.
 *
 * Primitive modes run the reference's classes directly:
 *   hash            Minimizer_Utility::hash          (include/Minimizer_Utility.hpp:97-107)
 *   min K L         Min_Iterator<K-1>::reset/advance  (include/Minimizer_Iterator.hpp:306-378)
 *   state F         State_Config<false>::update / edge_at / edge_count
 * The pipeline mode "run K L C G" drives those classes (Directed_Vertex,
 * State_Config, Unitig_Scratch, Maximal_Unitig_Scratch, FASTA_Record,
 * Character_Buffer) with the loops of src/Graph_Partitioner.cpp:461-597,
 * src/Subgraph.cpp:43-108 / 183-271 and include/Subgraph.hpp:414-543.
 * The loops are restated; every type, rolling step, canonical form, state
 * update, unitig finalisation and FASTA byte comes from the reference.
 */
#include "Minimizer_Iterator.hpp"
#include "Minimizer_Utility.hpp"
#include "State_Config.hpp"
#include "Directed_Vertex.hpp"
#include "Maximal_Unitig_Scratch.hpp"
#include "Character_Buffer.hpp"
#include "DNA_Utility.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

using cuttlefish::side_t;
using cuttlefish::base_t;

static std::vector<std::string> read_lines() {
    std::vector<std::string> v;
    std::string s;
    while (std::getline(std::cin, s)) v.push_back(s);
    return v;
}

template <uint16_t K1>   // K1 = k - 1
static void mode_min(uint16_t l) {
    for (const std::string& s : read_lines()) {
        if (s.size() < K1) { std::printf("\n"); continue; }
        Min_Iterator<K1> it(l);
        it.reset(s.c_str());
        std::printf("%llu", (unsigned long long)it.hash());
        for (size_t i = K1; i < s.size(); ++i) {
            it.advance(s[i]);
            std::printf(" %llu", (unsigned long long)it.hash());
        }
        std::printf("\n");
    }
}

static void mode_state(uint8_t fth) {
    cuttlefish::Edge_Frequency::set_edge_threshold(fth);
    for (const std::string& s : read_lines()) {
        unsigned ef, st; int front, back, s0, s1;
        if (std::sscanf(s.c_str(), "%u %u %d %d %d %d", &ef, &st, &front, &back, &s0, &s1) != 6) continue;
        cuttlefish::State_Config<false> c;
        static_assert(sizeof(c) == 8, "layout");
        uint32_t w[2] = {ef, st};
        std::memcpy(&c, w, 5);
        c.update(base_t(front), base_t(back), side_t(s0), side_t(s1));
        std::memcpy(w, &c, 5);
        std::printf("%u %u %d %d\n", w[0], w[1] & 0xFF, int(c.edge_at(side_t::front)), int(c.edge_at(side_t::back)));
    }
}

// ---------------------------------------------------------------------------
template <uint16_t k>
struct Pipeline {
    struct Rec { uint32_t g; uint8_t len, ld, rd; std::string lab; };
    typedef cuttlefish::State_Config<false> State;

    uint16_t l; uint64_t G; uint8_t fth;
    std::vector<std::vector<Rec>> bucket;
    std::vector<Rec> all;

    // insertion-ordered map, the iteration order of include/Subgraph.hpp:53
    std::vector<Kmer<k>> keys; std::vector<State> vals;
    std::map<std::string, size_t> index;   // keyed by the k-mer label

    size_t find(const Kmer<k>& x) { std::string s; x.get_label(s); auto it = index.find(s); return it == index.end() ? SIZE_MAX : it->second; }
    State& at(const Kmer<k>& x) {
        std::string s; x.get_label(s);
        auto it = index.find(s);
        if (it != index.end()) return vals[it->second];
        index.emplace(s, keys.size()); keys.push_back(x); vals.emplace_back();
        return vals.back();
    }

    void partition(const std::string& seq) {     // src/Graph_Partitioner.cpp:461-597
        const std::size_t sup_th = 2 * (k - 1) - l;
        std::string padded = seq; padded.resize(seq.size() + 32, '\0');
        const char* s = padded.c_str(); const std::size_t n = seq.size();
        std::size_t last = 0;
        while (true) {
            std::size_t fb, fl;
            for (fb = last; fb + (k + 1) <= n; ++fb) if (DNA_Utility::is_DNA_base(s[fb])) break;
            if (fb + (k + 1) > n) break;
            const char* frag = s + fb;
            for (fl = 1; fl < (k + 1); ++fl) if (!DNA_Utility::is_DNA_base(frag[fl])) break;
            if (fl < (k + 1)) { last = fb + fl; continue; }
            Min_Iterator<k - 1> it(l);
            std::size_t cur_off = 0, idx = 0; fl = k - 1;
            it.reset(frag);
            uint64_t cur_g = it.hash() & (G - 1), prev_g = G, next_g;
            auto emit = [&](uint64_t g, std::size_t off, std::size_t len, bool ld, bool rd) {
                Rec r{(uint32_t)g, (uint8_t)len, ld, rd, std::string(frag + off, len)};
                all.push_back(r); bucket[g].push_back(r);
            };
            while (DNA_Utility::is_DNA_base(frag[fl])) {
                const std::size_t len = idx + (k - 1);
                it.advance(frag[fl]); idx++, fl++;
                next_g = it.hash() & (G - 1);
                if (next_g != cur_g || len == sup_th) {
                    const bool lj = cur_off > 0;
                    emit(cur_g, cur_off - lj, lj + len + 1, lj && prev_g != cur_g, next_g != cur_g);
                    cur_off += idx; prev_g = cur_g; cur_g = next_g; idx = 0;
                }
            }
            const std::size_t len = fl - cur_off; const bool lj = cur_off > 0;
            emit(cur_g, cur_off - lj, lj + len, lj && prev_g != cur_g, false);
            last = fb + fl;
        }
    }

    static base_t base_of(char c) { return DNA_Utility::map_base(c); }

    void construct(const std::vector<Rec>& recs) {     // src/Subgraph.cpp:43-108
        keys.clear(); vals.clear(); index.clear();
        for (const Rec& r : recs) {
            const std::size_t len = r.len;
            Directed_Vertex<k> v(Kmer<k>(r.lab.c_str()));
            Kmer<k> pred_v;
            std::size_t i = 0;
            while (true) {
                const bool canon = v.in_canonical_form();
                const base_t pred = (i == 0 ? base_t::E : base_of(r.lab[i - 1]));
                const base_t succ = (i + k == len ? base_t::E : base_of(r.lab[i + k]));
                base_t front = canon ? pred : DNA_Utility::complement(succ);
                base_t back = canon ? succ : DNA_Utility::complement(pred);
                if (i > 0 && v.canonical() == pred_v) (canon ? front : back) = base_t::E;
                State& st = at(v.canonical());
                st.update_edges(front, back);
                if (i == 0 && r.ld) st.mark_discontinuous(v.entrance_side());
                if (i + k == len && r.rd) st.mark_discontinuous(v.exit_side());
                if (i + k == len) break;
                pred_v = v.canonical();
                v.roll_forward(succ);
                i++;
            }
        }
    }

    enum Term { T_NULL, T_BRANCHED, T_CROSSED, T_DEAD, T_EXIT };

    Term walk(const Kmer<k>& v_hat, side_t s_hat, Unitig_Scratch<k>& u, Directed_Vertex<k>& exit_v) {  // include/Subgraph.hpp:467-543
        const side_t s_icc_return = cuttlefish::inv_side(s_hat);
        Directed_Vertex<k> v(s_hat == side_t::back ? v_hat : v_hat.reverse_complement());
        side_t s_v = s_hat;
        size_t it = find(v.canonical());
        State state = vals[it];
        u.init(v);
        while (true) {
            vals[it].mark_visited();
            base_t b = state.edge_at(s_v);
            if (b == base_t::N) return T_BRANCHED;
            if (b == base_t::E) { if (!state.is_discontinuous(s_v)) return T_DEAD; exit_v = v; return T_EXIT; }
            if (s_v == side_t::front) b = DNA_Utility::complement(b);
            v.roll_forward(b);
            it = find(v.canonical());
            state = vals[it];
            s_v = v.entrance_side();
            if (state.is_branching_side(s_v)) return T_CROSSED;
            if (state.is_visited()) { if (v.canonical() == v_hat && s_v == s_icc_return) u.mark_cycle(); return T_CROSSED; }
            u.extend(v, DNA_Utility::map_char(b));
            s_v = cuttlefish::opposite_side(s_v);
        }
    }

    void contract(uint32_t g, Character_Buffer<std::ofstream>& fa, std::FILE* lm) {   // src/Subgraph.cpp:183-271
        Maximal_Unitig_Scratch<k> mu;
        for (size_t p = 0; p < keys.size(); ++p) {
            const Kmer<k> v = keys[p];
            const State& st = vals[p];
            if (st.is_visited()) continue;
            if (st.is_isolated()) { std::printf("P %u\n", g); continue; }
            mu.mark_linear();
            Directed_Vertex<k> v_l, v_r;
            Term end_l = T_NULL, end_r;
            end_r = walk(v, side_t::back, mu.unitig(side_t::back), v_r);
            if (mu.unitig(side_t::back).is_cycle()) mu.mark_cycle(side_t::back);
            else end_l = walk(v, side_t::front, mu.unitig(side_t::front), v_l);
            if (end_l == T_EXIT || end_r == T_EXIT) {
                mu.finalize_weak();
                const auto& uf = mu.unitig_label(side_t::front);
                const auto& ub = mu.unitig_label(side_t::back);
                std::string lab(uf); lab.append(ub, k, std::string::npos);
                std::string su, sv;
                (end_l == T_EXIT ? v_l.canonical() : Kmer<k>(std::string(k, 'T'))).get_label(su);
                (end_r == T_EXIT ? v_r.canonical() : Kmer<k>(std::string(k, 'T'))).get_label(sv);
                const int fu = (end_l == T_EXIT ? (v_l.entrance_side() == side_t::back) : 1);
                const int fv = (end_r == T_EXIT ? (v_r.entrance_side() == side_t::back) : 1);
                std::fprintf(lm, "%u %s %s %s %d\n", g, lab.c_str(), su.c_str(), sv.c_str(),
                             fu | (fv << 1) | ((end_l != T_EXIT) << 2) | ((end_r != T_EXIT) << 3));
            } else {
                mu.finalize();
                mu.add_fasta_rec_to_buffer(fa);
                std::printf("T %u %d\n", g, (int)mu.is_cycle());
            }
        }
        for (size_t p = 0; p < keys.size(); ++p) {
            std::string s; keys[p].get_label(s);
            uint32_t w[2] = {0, 0}; std::memcpy(w, &vals[p], 5);
            std::printf("V %u %s %u %u\n", g, s.c_str(), w[0], w[1] & 0xFF);
        }
    }

    void run(const char* fa_path, const char* lm_path) {
        cuttlefish::Edge_Frequency::set_edge_threshold(fth);
        bucket.assign(G, {});
        for (const std::string& s : read_lines()) partition(s);
        for (const Rec& r : all) std::printf("R %u %u %d %d %s\n", r.g, (unsigned)r.len, (int)r.ld, (int)r.rd, r.lab.c_str());
        std::ofstream fa(fa_path);
        std::FILE* lm = std::fopen(lm_path, "w");
        {
            Character_Buffer<std::ofstream> buf(fa);
            for (uint32_t g = 0; g < G; ++g) {
                if (bucket[g].empty()) continue;
                construct(bucket[g]);
                contract(g, buf, lm);
            }
        }
        std::fclose(lm);
    }
};

template <uint16_t k>
static int run_k(int argc, char** argv) {
    Pipeline<k> p;
    p.l = (uint16_t)std::atoi(argv[3]); p.fth = (uint8_t)std::atoi(argv[4]); p.G = std::strtoull(argv[5], nullptr, 10);
    p.run(argv[6], argv[7]);
    (void)argc;
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string m = argv[1];
    if (m == "hash") {
        for (const std::string& s : read_lines())
            std::printf("%llu\n", (unsigned long long)Minimizer_Utility::hash(std::strtoull(s.c_str(), nullptr, 10)));
        return 0;
    }
    if (m == "state") { mode_state((uint8_t)std::atoi(argv[2])); return 0; }
    if (m == "min") {
        const int k = std::atoi(argv[2]); const uint16_t l = (uint16_t)std::atoi(argv[3]);
        switch (k) {
            case 3: mode_min<2>(l); break;   case 7: mode_min<6>(l); break;
            case 5: mode_min<4>(l); break;   case 9: mode_min<8>(l); break;
            case 15: mode_min<14>(l); break; case 23: mode_min<22>(l); break;
            case 31: mode_min<30>(l); break; case 63: mode_min<62>(l); break;
            case 95: mode_min<94>(l); break; case 127: mode_min<126>(l); break;
            default: return 3;
        }
        return 0;
    }
    if (m == "run" && argc >= 8) {   // run K L C G fasta_out lmtig_out  < records (one per line)
        switch (std::atoi(argv[2])) {
            case 3: return run_k<3>(argc, argv);   case 7: return run_k<7>(argc, argv);
            case 5: return run_k<5>(argc, argv);   case 9: return run_k<9>(argc, argv);
            case 15: return run_k<15>(argc, argv); case 23: return run_k<23>(argc, argv);
            case 31: return run_k<31>(argc, argv); case 63: return run_k<63>(argc, argv);
            case 95: return run_k<95>(argc, argv); case 127: return run_k<127>(argc, argv);
            default: return 3;
        }
    }
    return 2;
}
