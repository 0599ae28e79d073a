// cfg_collate.cpp -- joins the lm-tigs of a run into global maximal unitigs (host).
//
// This is the job of the reference's discontinuity-graph phases
// (Discontinuity_Graph_Contractor::contract, Contracted_Graph_Expander::expand,
// Unitig_Collator::collate; src/Discontinuity_Graph_Contractor.cpp,
// src/Contracted_Graph_Expander.cpp, src/Unitig_Collator.cpp), done directly:
// every lm-tig is an edge of the discontinuity graph between (u, s_u) and
// (v, s_v), a discontinuity vertex carries at most one lm-tig on each side (its
// two appearances, one per subgraph), and a maximal unitig is a maximal chain of
// lm-tigs glued k bases deep at those vertices (a closed chain is a cycle).
// Labels are oriented as Unitig_Collator does: a linear unitig starts with the
// smaller of its first k-mer and the reverse complement of its last k-mer
// (Maximal_Unitig::canonicalize, include/Unitig_Collator.hpp:308-347); a cycle
// starts at its smallest k-mer over both strands, in that strand
// (canonicalize_cycle, :367-407).  Records are ">0\nSEQ\n" (src/Unitig_Collator.cpp:334-335).
#include "cuttlefish_gpu.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

namespace {

struct End {          // one non-phi end of an lm-tig
    uint64_t w[4];    // canonical k-mer, words as in cfg_lmtig::u
    uint32_t side;    // attachment side: 0 front, 1 back
    uint32_t id;      // lm-tig index << 1 | end (0 = u, 1 = v)
    bool same_vertex(const End& o) const { return std::memcmp(w, o.w, sizeof w) == 0; }
    bool operator<(const End& o) const {
        for (int j = 3; j >= 0; --j)
            if (w[j] != o.w[j]) return w[j] < o.w[j];
        return side < o.side;
    }
};
End end_of(const uint64_t* key, uint32_t side, uint32_t id) {
    End e;
    std::memcpy(e.w, key, sizeof e.w);
    e.side = side; e.id = id;
    return e;
}

inline char comp(char c) { return c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'A'; }

void append_oriented(std::string& out, const char* lab, uint32_t len, bool fwd, uint32_t skip) {
    if (fwd) out.append(lab + skip, len - skip);
    else
        for (int64_t i = (int64_t)len - 1 - skip; i >= 0; --i) out.push_back(comp(lab[i]));
}

// linear: the smaller of S and its reverse complement, decided on the first k bases
void canonical_linear(std::string& s, uint32_t k) {
    const size_t n = s.size();
    for (size_t i = 0; i < k && i < n; ++i) {
        const char f = s[i], b = comp(s[n - 1 - i]);
        if (f < b) return;
        if (f > b) {
            std::string r(n, 'A');
            for (size_t j = 0; j < n; ++j) r[j] = comp(s[n - 1 - j]);
            s.swap(r);
            return;
        }
    }
}

// cycle: s holds the n+k-1 bases of a cycle of n k-mers (its last k-1 bases repeat its
// first k-1); start at the smallest k-mer over both strands, in that strand.
void canonical_cycle(std::string& s, uint32_t k) {
    const size_t L = s.size(), n = L - k + 1;
    std::string r(L, 'A');
    for (size_t j = 0; j < L; ++j) r[j] = comp(s[L - 1 - j]);
    size_t best_i = 0; bool best_rc = false;
    const char* bp = s.data();
    for (size_t i = 0; i < n; ++i) {
        if (std::memcmp(s.data() + i, bp, k) < 0) { bp = s.data() + i; best_i = i; best_rc = false; }
        if (std::memcmp(r.data() + i, bp, k) < 0) { bp = r.data() + i; best_i = i; best_rc = true; }
    }
    const std::string& src = best_rc ? r : s;
    std::string out;
    out.reserve(L);
    out.append(src, best_i, std::string::npos);          // from the smallest k-mer to the end
    out.append(src, k - 1, best_i);                       // wrap around past the k-1 overlap
    s.swap(out);
}

}  // namespace

extern "C" int cfg_collate_lmtigs(uint32_t k, const cfg_lmtig* lm, uint64_t n_lm, const char* text,
                                  char** out, uint64_t* out_bytes, uint64_t* n_unitigs, uint64_t* n_cycles) {
    if (!out || !out_bytes || (n_lm && (!lm || !text)) || k < 3 || k > 127 || n_lm >= (1ull << 31)) return CFG_ERR_BAD_INPUT;
    std::vector<End> ends;
    ends.reserve(2 * n_lm);
    for (uint64_t i = 0; i < n_lm; ++i) {
        const uint8_t f = lm[i].flags;
        if (!(f & 4)) ends.push_back(end_of(lm[i].u, (uint32_t)(f & 1), (uint32_t)(i << 1)));
        if (!(f & 8)) ends.push_back(end_of(lm[i].v, (uint32_t)((f >> 1) & 1), (uint32_t)((i << 1) | 1)));
    }
    std::sort(ends.begin(), ends.end());
    // partner of each end: the other side of the same vertex
    std::vector<uint32_t> partner(2 * n_lm, 0xffffffffu);
    for (size_t a = 0; a < ends.size();) {
        size_t b = a;
        while (b < ends.size() && ends[b].same_vertex(ends[a])) ++b;
        if (b - a > 2 || (b - a == 2 && ends[a].side == ends[a + 1].side)) return CFG_ERR_STATE;   // not a valid graph
        if (b - a == 2) { partner[ends[a].id] = ends[a + 1].id; partner[ends[a + 1].id] = ends[a].id; }
        a = b;
    }
    std::vector<uint8_t> done(n_lm, 0);
    std::string res;
    uint64_t units = 0, cycles = 0;
    std::string s;
    auto emit = [&](std::string& lab) { res += ">0\n"; res += lab; res += '\n'; ++units; };
    auto terminal = [&](uint32_t end_id) {   // phi, or no lm-tig on the vertex's other side
        const uint8_t f = lm[end_id >> 1].flags;
        const bool phi = (end_id & 1) ? (f & 8) : (f & 4);
        return phi || partner[end_id] == 0xffffffffu;
    };
    auto walk = [&](uint32_t start_end, bool cycle) {
        s.clear();
        uint32_t e = start_end;   // the end we enter the current lm-tig by
        bool first = true;
        for (uint64_t guard = 0; guard <= n_lm; ++guard) {
            const uint32_t i = e >> 1;
            const bool fwd = (e & 1) == 0;   // entered by u: read the label forward
            if (done[i]) break;              // back at the start of a cycle
            done[i] = 1;
            append_oriented(s, text + lm[i].label_off, lm[i].label_len, fwd, first ? 0 : k);
            first = false;
            const uint32_t out_end = e ^ 1;
            if (!cycle && terminal(out_end)) break;
            if (partner[out_end] == 0xffffffffu) break;
            e = partner[out_end];
        }
    };
    for (uint64_t i = 0; i < n_lm; ++i) {
        if (done[i]) continue;
        const uint32_t u_end = (uint32_t)(i << 1), v_end = u_end | 1;
        if (terminal(u_end)) walk(u_end, false);
        else if (terminal(v_end)) walk(v_end, false);
        else continue;
        canonical_linear(s, k);
        emit(s);
    }
    for (uint64_t i = 0; i < n_lm; ++i) {   // what is left closes on itself
        if (done[i]) continue;
        walk((uint32_t)(i << 1), true);
        // the label ends with its first k-mer again: keep the n+k-1 bases of the cycle
        if (s.size() < k) return CFG_ERR_STATE;
        s.pop_back();
        canonical_cycle(s, k);
        emit(s);
        ++cycles;
    }
    char* buf = (char*)std::malloc(res.size() + 1);
    if (!buf) return CFG_ERR_OOM;
    std::memcpy(buf, res.data(), res.size());
    buf[res.size()] = 0;
    *out = buf;
    *out_bytes = res.size();
    if (n_unitigs) *n_unitigs = units;
    if (n_cycles) *n_cycles = cycles;
    return CFG_OK;
}

extern "C" void cfg_free(void* p) { std::free(p); }
