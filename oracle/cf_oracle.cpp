/*
 * cf_oracle.cpp -- CPU restatement of Cuttlefish's compaction hot path
 * (partition -> per-subgraph construct -> local unitig walk).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA path.  Nothing in
 * the product links, loads or calls this file.
 *
 * Every function cites the reference file:line it restates.  Disk buckets,
 * lz4, parlay workers and spdlog sinks are replaced by in-memory vectors and
 * std::thread; the per-subgraph map keeps insertion order, which is the order
 * the reference's ankerl::unordered_dense map iterates in
 * (include/Subgraph.hpp:53), so the local walk visits seeds exactly as the
 * reference does for a single input file.
 */
#include "cf_oracle.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace orc {

// ---------------------------------------------------------------------------
// DNA coding: A0 C1 G2 T3, N4 (branching), E5 (empty)  -- include/DNA.hpp:16-24
constexpr uint8_t A = 0, C = 1, G = 2, T = 3, N = 4, E = 5;
enum Side : uint8_t { FRONT = 0, BACK = 1, UNSPEC = 2 };  // include/globals.hpp:70-80

static inline uint8_t comp(uint8_t b) { return b < 4 ? (uint8_t)(3 - b) : b; }  // DNA_Utility.hpp COMPLEMENTED_BASE
// is_DNA_base: (c & 0x5F) in {A,C,G,T}  -- include/DNA_Utility.hpp:167-172.  Bytes >= 0x80 are not bases here.
static inline bool is_dna(unsigned char c) {
    if (c & 0x80) return false;
    const unsigned char u = c & 0x5F;
    return u == 'A' || u == 'C' || u == 'G' || u == 'T';
}
// map_base_unchecked -- include/DNA_Utility.hpp:121-124
static inline uint8_t map_base(unsigned char c) { return (uint8_t)(((c >> 2) ^ (c >> 1)) & 3); }
static const char CHR[4] = {'A', 'C', 'G', 'T'};

// ---------------------------------------------------------------------------
// wyhash v4.2 (public domain, W. Yi), restated for an 8-byte little-endian key
// with WYHASH_CONDOM=1 and the 128-bit mum: include/wyhash/wyhash.h:47-142.
// Salt: include/Minimizer_Utility.hpp:26.
static const uint64_t SALT[4] = {4167021922371662411ull, 7320285940802167691ull,
                                 14307255741305819987ull, 10859488101230029397ull};
static inline void mum(uint64_t& a, uint64_t& b) {
    const __uint128_t r = (__uint128_t)a * b;
    a = (uint64_t)r;
    b = (uint64_t)(r >> 64);
}
static inline uint64_t mix(uint64_t a, uint64_t b) { mum(a, b); return a ^ b; }
static inline uint64_t wyhash8(uint64_t x) {
    const uint64_t seed = mix(0 ^ SALT[0], SALT[1]);       // seed ^= wymix(seed^s0, s1), seed 0
    const uint64_t lo = (uint32_t)x, hi = x >> 32;
    uint64_t a = (lo << 32) | hi;                          // (r4(p)<<32) | r4(p+4)
    uint64_t b = (hi << 32) | lo;                          // (r4(p+4)<<32) | r4(p)
    a ^= SALT[1];
    b ^= seed;
    mum(a, b);
    return mix(a ^ SALT[0] ^ 8, b ^ SALT[1]);
}

// Canonical l-mer hash: Min_Iterator::lmer_hash -- include/Minimizer_Iterator.hpp:291-296
static inline uint64_t lmer_hash(uint64_t lmer, uint64_t lmer_bar) {
    return std::min(wyhash8(lmer), wyhash8(lmer_bar));
}

// l-minimizer hash of each (k-1)-mer of s[0..n): Min_Iterator<k-1>::reset/advance/hash,
// include/Minimizer_Iterator.hpp:306-378.  The two-stack window there returns the minimum
// of the (k-1)-l+1 l-mer hashes of the window; the minimum is restated directly.
static void km1_min_hashes(const unsigned char* s, uint64_t n, uint32_t k, uint32_t l, uint64_t* out) {
    const uint32_t K = k - 1;
    if (n < K) return;
    const uint64_t n_l = n - l + 1;
    std::vector<uint64_t> H(n_l);
    const uint64_t mask = (l == 32) ? ~0ull : ((1ull << (2 * l)) - 1);
    uint64_t fw = 0, rc = 0;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t b = map_base(s[i]);
        fw = ((fw << 2) | b) & mask;                                 // last_lmer roll (:372)
        rc = (rc >> 2) | ((3 - b) << (2 * (l - 1)));                 // last_lmer_bar roll (:373)
        if (i + 1 >= l) H[i + 1 - l] = lmer_hash(fw, rc);
    }
    const uint32_t w = K - l + 1;                                    // l-mers per (k-1)-mer
    for (uint64_t j = 0; j + K <= n; ++j) {
        uint64_t m = ~0ull;
        for (uint32_t t = 0; t < w; ++t) m = std::min(m, H[j + t]);
        out[j] = m;
    }
}

// ---------------------------------------------------------------------------
// Kmer<k>: kmer_data[0] holds the last 32 bases, last base in bits 1:0, and word j the
// 32 before word j-1's (include/Kmer.hpp:45-54); words compare high to low (:509-521).
// Four words hold any k <= 127 (INSTANCE_COUNT 64, include/globals.hpp:16-22); words
// past ceil(k/32) stay 0.
constexpr int KW = 4;
struct Kmer {
    uint64_t w[KW];  // w[0] low ... w[KW-1] high
    bool operator==(const Kmer& o) const { return std::memcmp(w, o.w, sizeof w) == 0; }
    bool operator<(const Kmer& o) const {
        for (int j = KW - 1; j > 0; --j)
            if (w[j] != o.w[j]) return w[j] < o.w[j];
        return w[0] < o.w[0];
    }
};

struct KCodec {
    uint32_t k;
    uint64_t m[KW];  // the bits each word holds
    explicit KCodec(uint32_t k_) : k(k_) {
        for (int j = 0; j < KW; ++j) {
            const int left = 2 * (int)k - 64 * j;
            m[j] = left >= 64 ? ~0ull : left <= 0 ? 0ull : ((1ull << left) - 1);
        }
    }
    // roll_to_next_kmer: shift one base in at the end -- include/Kmer.hpp:610-621
    void push_back(Kmer& x, uint8_t b) const {
        for (int j = KW - 1; j > 0; --j) x.w[j] = ((x.w[j] << 2) | (x.w[j - 1] >> 62)) & m[j];
        x.w[0] = ((x.w[0] << 2) | b) & m[0];
    }
    // reverse-complement roll: shift one complemented base in at the front
    void push_front(Kmer& x, uint8_t b) const {
        const uint32_t pos = 2 * (k - 1);
        for (int j = 0; j < KW - 1; ++j) x.w[j] = (x.w[j] >> 2) | (x.w[j + 1] << 62);
        x.w[KW - 1] >>= 2;
        x.w[pos / 64] |= (uint64_t)b << (pos % 64);
    }
    uint8_t base_at(const Kmer& x, uint32_t i) const {  // i-th base from the start
        const uint32_t bitpos = 2 * (k - 1 - i);
        return (uint8_t)((x.w[bitpos / 64] >> (bitpos % 64)) & 3);
    }
    Kmer rc(const Kmer& x) const {
        Kmer r{};
        for (uint32_t i = 0; i < k; ++i) push_back(r, (uint8_t)(3 - base_at(x, k - 1 - i)));
        return r;
    }
    std::string label(const Kmer& x) const {
        std::string s(k, 'A');
        for (uint32_t i = 0; i < k; ++i) s[i] = CHR[base_at(x, i)];
        return s;
    }
};

// Directed_Vertex<k> -- include/Directed_Vertex.hpp:20-321
struct DVertex {
    Kmer fw, bw;
    bool canon_fw;  // &kmer_ == kmer_hat_ptr; Kmer::canonical picks kmer if kmer < rev_compl (:687-690)
    const Kmer& canonical() const { return canon_fw ? fw : bw; }
    Side entrance_side() const { return canon_fw ? FRONT : BACK; }  // :301-306
    Side exit_side() const { return canon_fw ? BACK : FRONT; }      // :295-299
};
static inline void dv_init(const KCodec& kc, DVertex& v, const Kmer& x) {
    v.fw = x; v.bw = kc.rc(x); v.canon_fw = v.fw < v.bw;
}
static inline void dv_roll(const KCodec& kc, DVertex& v, uint8_t b) {  // roll_forward
    kc.push_back(v.fw, b);
    kc.push_front(v.bw, (uint8_t)(3 - b));
    v.canon_fw = v.fw < v.bw;
}

// ---------------------------------------------------------------------------
// State_Config<false> -- include/State_Config.hpp:24-268, src/State_Config.cpp:8-13
struct State {
    uint32_t ef = 0;
    uint8_t st = 0;  // bit0 visited, bit1 disc front, bit2 disc back (:103-104)
};
static inline void add_edge(uint32_t& ef, Side s, uint8_t e) {  // Edge_Frequency::add_edge (:207-217)
    const uint32_t off = (s == FRONT ? 0 : 16) + 4 * e;
    const uint32_t f = (ef >> off) & 0xF;
    if (f < 15) ef = (ef & ~(0xFu << off)) | ((f + 1) << off);
}
static inline void update_edges(State& s, uint8_t front, uint8_t back) {  // Vertex_Neighborhood::update_edges
    if (front != E) add_edge(s.ef, FRONT, front);
    if (back != E) add_edge(s.ef, BACK, back);
}
static inline void mark_disc(State& s, Side side) { s.st |= (side == FRONT ? 2 : 4); }
static inline bool is_disc(const State& s, Side side) { return s.st & (side == FRONT ? 2 : 4); }
static inline bool visited(const State& s) { return s.st & 1; }
static inline uint32_t edge_count(uint32_t ef, Side s, uint32_t fth) {  // :220-229
    const uint32_t off = s == FRONT ? 0 : 16;
    uint32_t c = 0;
    for (int b = 0; b < 4; ++b) c += (((ef >> (off + 4 * b)) & 0xF) >= fth);
    return c;
}
static inline uint8_t edge_at(uint32_t ef, Side s, uint32_t fth) {  // :232-252
    const uint32_t off = s == FRONT ? 0 : 16;
    uint32_t c = 0; uint8_t last = E;
    for (int b = 0; b < 4; ++b)
        if (((ef >> (off + 4 * b)) & 0xF) >= fth) { ++c; last = (uint8_t)b; }
    return c == 0 ? E : (c == 1 ? last : N);
}

// ---------------------------------------------------------------------------
// Insertion-ordered map Kmer -> State (dense vector + open-addressed index).
struct OMap {
    std::vector<Kmer> keys;
    std::vector<State> vals;
    std::vector<int64_t> idx;
    uint64_t mask = 0;
    static uint64_t h(const Kmer& x) {
        uint64_t z = x.w[0] * 0x9E3779B97F4A7C15ull ^ (x.w[1] + 0x632BE59BD9B4E019ull) ^ (x.w[2] * 0xC2B2AE3D27D4EB4Full) ^
                     (x.w[3] * 0x165667B19E3779F9ull);
        z ^= z >> 31; z *= 0xBF58476D1CE4E5B9ull; z ^= z >> 29;
        return z;
    }
    void clear() { keys.clear(); vals.clear(); idx.assign(1024, -1); mask = 1023; }
    void grow() {
        std::vector<int64_t> n((mask + 1) * 2, -1);
        const uint64_t nm = n.size() - 1;
        for (size_t i = 0; i < keys.size(); ++i) {
            uint64_t p = h(keys[i]) & nm;
            while (n[p] >= 0) p = (p + 1) & nm;
            n[p] = (int64_t)i;
        }
        idx.swap(n); mask = nm;
    }
    int64_t find(const Kmer& x) const {
        uint64_t p = h(x) & mask;
        while (idx[p] >= 0) { if (keys[idx[p]] == x) return idx[p]; p = (p + 1) & mask; }
        return -1;
    }
    State& operator[](const Kmer& x) {  // HT[kmer]: find or default-insert
        if ((keys.size() + 1) * 2 > mask + 1) grow();
        uint64_t p = h(x) & mask;
        while (idx[p] >= 0) { if (keys[idx[p]] == x) return vals[idx[p]]; p = (p + 1) & mask; }
        idx[p] = (int64_t)keys.size();
        keys.push_back(x); vals.emplace_back();
        return vals.back();
    }
};

// ---------------------------------------------------------------------------
struct Rec {      // a weak super k-mer: Super_Kmer_Attributes<false> + label (include/Super_Kmer_Attributes.hpp:25-61)
    uint32_t g;
    uint8_t len, flags;  // flags bit0 l_disc, bit1 r_disc
    uint64_t src;        // offset in the input concatenation
};

// Unitig_Scratch<k> -- include/Unitig_Scratch.hpp:18-189
struct UScratch {
    DVertex anchor, endpoint, min_vertex;
    size_t vertex_idx = 0, min_v_idx = 0, size = 0;
    std::string label;
    bool cycle = false;
    void init(const KCodec& kc, const DVertex& v) {
        anchor = endpoint = min_vertex = v;
        vertex_idx = min_v_idx = 0; size = 1;
        label = kc.label(v.fw);
        cycle = false;
    }
    bool extend(const DVertex& v, char b) {
        if (v.canonical() == anchor.canonical()) { cycle = true; return false; }
        endpoint = v;
        ++vertex_idx; ++size;
        if (v.canonical() < min_vertex.canonical()) { min_vertex = v; min_v_idx = vertex_idx; }
        label.push_back(b);
        return true;
    }
    void reverse_complement() {
        std::string r(label.rbegin(), label.rend());
        for (char& c : r) c = CHR[3 - map_base((unsigned char)c)];
        label.swap(r);
        min_v_idx = size - 1 - min_v_idx;
    }
};

enum Term { T_NULL, T_BRANCHED, T_CROSSED, T_DEAD, T_EXIT };  // Walk_Termination, include/Subgraph.hpp:362-369

struct SubOut {
    std::string fasta;
    std::string lm_text;
    std::vector<uint64_t> lm_len;
    std::vector<Kmer> lm_u, lm_v;
    std::vector<uint8_t> lm_flags;
    std::vector<Kmer> vkeys;
    std::vector<State> vstates;
    uint64_t n_inst = 0, n_isolated = 0, n_phantom = 0, n_trivial = 0, n_icc = 0, n_lmtig = 0, n_edges = 0;
};

struct Worker {
    const KCodec& kc;
    uint32_t k, fth;
    OMap M;
    Worker(const KCodec& kc_, uint32_t fth_) : kc(kc_), k(kc_.k), fth(fth_) {}

    // Subgraph::construct -- src/Subgraph.cpp:43-108
    void construct(const std::vector<Rec>& recs, const std::string& in, SubOut& o) {
        M.clear();
        for (const Rec& r : recs) {
            const unsigned char* lab = (const unsigned char*)in.data() + r.src;
            const uint32_t len = r.len;
            o.n_inst += len - (k - 1);
            Kmer x{};
            for (uint32_t i = 0; i < k; ++i) kc.push_back(x, map_base(lab[i]));
            DVertex v; dv_init(kc, v, x);
            Kmer pred_v{};
            for (uint32_t idx = 0;; ++idx) {
                const bool canon = v.canon_fw;
                const uint8_t pred = idx == 0 ? E : map_base(lab[idx - 1]);
                const uint8_t succ = idx + k == len ? E : map_base(lab[idx + k]);
                uint8_t front = canon ? pred : comp(succ);
                uint8_t back = canon ? succ : comp(pred);
                if (idx > 0 && v.canonical() == pred_v) (canon ? front : back) = E;  // self-loop (:82-83)
                o.n_edges += (succ != E);
                State& st = M[v.canonical()];                                      // HT_Router::update
                update_edges(st, front, back);
                if (idx == 0 && (r.flags & 1)) mark_disc(st, v.entrance_side());
                if (idx + k == len && (r.flags & 2)) mark_disc(st, v.exit_side());
                if (idx + k == len) break;
                pred_v = v.canonical();
                dv_roll(kc, v, succ);
            }
        }
    }

    // Subgraph::walk_unitig -- include/Subgraph.hpp:467-543
    Term walk(const Kmer& v_hat, Side s_hat, UScratch& u, DVertex& exit_v) {
        const Side s_icc_return = s_hat == BACK ? FRONT : BACK;
        DVertex v; dv_init(kc, v, s_hat == BACK ? v_hat : kc.rc(v_hat));
        Side s_v = s_hat;
        int64_t it = M.find(v.canonical());
        State state = M.vals[it];
        u.init(kc, v);
        while (true) {
            M.vals[it].st |= 1;  // mark_visited
            uint8_t b = edge_at(state.ef, s_v, fth);
            if (b == N) return T_BRANCHED;
            if (b == E) {
                if (!is_disc(state, s_v)) return T_DEAD;
                exit_v = v;
                return T_EXIT;
            }
            if (s_v == FRONT) b = comp(b);
            dv_roll(kc, v, b);
            it = M.find(v.canonical());
            state = M.vals[it];
            s_v = v.entrance_side();
            if (edge_count(state.ef, s_v, fth) > 1) return T_CROSSED;  // is_branching_side
            if (visited(state)) {
                if (v.canonical() == v_hat && s_v == s_icc_return) u.cycle = true;
                return T_CROSSED;
            }
            u.extend(v, CHR[b]);
            s_v = s_v == FRONT ? BACK : FRONT;
        }
    }

    // Subgraph::contract + extract_maximal_unitig -- src/Subgraph.cpp:183-271, include/Subgraph.hpp:414-464
    void contract(SubOut& o) {
        UScratch ub, uf;
        for (size_t p = 0; p < M.keys.size(); ++p) {
            const Kmer v = M.keys[p];
            const State vs = M.vals[p];
            if (visited(vs)) continue;
            if (edge_count(vs.ef, FRONT, fth) == 0 && edge_count(vs.ef, BACK, fth) == 0) {  // is_isolated
                if (vs.st & 6) o.n_phantom++;
                o.n_isolated++;
                continue;
            }
            DVertex v_l, v_r;
            Term end_l = T_NULL, end_r;
            UScratch* cyc = nullptr;
            end_r = walk(v, BACK, ub, v_r);
            if (ub.cycle) cyc = &ub;
            else end_l = walk(v, FRONT, uf, v_l);
            if (end_l == T_EXIT || end_r == T_EXIT) {
                // finalize_weak (include/Maximal_Unitig_Scratch.hpp:225-233) + add_edge
                // (include/Discontinuity_Graph.hpp:143-151, include/Unitig_File.hpp:338-359)
                uf.reverse_complement();
                o.lm_text += uf.label;
                o.lm_text.append(ub.label, k, std::string::npos);
                o.lm_len.push_back(uf.label.size() + ub.label.size() - k);
                const Kmer phi = phi_kmer();
                o.lm_u.push_back(end_l == T_EXIT ? v_l.canonical() : phi);
                o.lm_v.push_back(end_r == T_EXIT ? v_r.canonical() : phi);
                const Side s_u = end_l == T_EXIT ? v_l.entrance_side() : BACK;
                const Side s_v = end_r == T_EXIT ? v_r.entrance_side() : BACK;
                o.lm_flags.push_back((uint8_t)((s_u == BACK) | ((s_v == BACK) << 1) |
                                               ((end_l != T_EXIT) << 2) | ((end_r != T_EXIT) << 3)));
                o.n_lmtig++;
            } else {
                o.n_trivial++;
                o.fasta += ">0\n";
                if (cyc) {
                    o.n_icc++;
                    // finalize (:213-221) + Character_Buffer::rotate_append_cycle (include/Character_Buffer.hpp:166-175)
                    if (!cyc->min_vertex.canon_fw) cyc->reverse_complement();
                    const std::string& s = cyc->label;
                    const size_t piv = cyc->min_v_idx;
                    o.fasta.append(s, piv, std::string::npos);
                    o.fasta.append(s, k - 1, piv);
                } else {
                    // finalize (:200-212) + fasta_rec (:243-248): orient so the label is canonical
                    const Kmer fb = uf.endpoint.bw, bb = ub.endpoint.bw;  // endpoint().kmer_bar()
                    if (fb < bb) {
                        uf.reverse_complement();
                        o.fasta += uf.label;
                        o.fasta.append(ub.label, k, std::string::npos);
                    } else {
                        ub.reverse_complement();
                        // after the swap: front = old back (rc'd), back = old front
                        if (bb < fb) { o.fasta += ub.label; o.fasta.append(uf.label, k, std::string::npos); }
                        else { o.fasta += uf.label; o.fasta.append(ub.label, k, std::string::npos); }
                    }
                }
                o.fasta += "\n";
            }
        }
        o.vkeys = M.keys;
        o.vstates = M.vals;
    }

    Kmer phi_kmer() const {  // all-T k-mer, include/Discontinuity_Graph.hpp:44-49
        Kmer x{};
        for (uint32_t i = 0; i < k; ++i) kc.push_back(x, T);
        return x;
    }
};

}  // namespace orc

using namespace orc;

struct orc_ctx {
    orc_params p;
    KCodec kc;
    std::string input;
    std::vector<Rec> recs;
    // flattened results
    std::vector<uint32_t> rec_g; std::vector<uint8_t> rec_len, rec_flags; std::vector<uint64_t> rec_src;
    std::vector<uint32_t> vtx_g; std::vector<uint64_t> vtx_key; std::vector<uint32_t> vtx_ef; std::vector<uint8_t> vtx_status;
    std::string fasta, lm_text;
    std::vector<uint64_t> lm_off, lm_u, lm_v; std::vector<uint8_t> lm_flags; std::vector<uint32_t> lm_g;
    uint64_t n_inst = 0, n_vert = 0, n_iso = 0, n_phan = 0, n_triv = 0, n_icc = 0, n_lm = 0, n_edges = 0;
    explicit orc_ctx(const orc_params& p_) : p(p_), kc(p_.k) {}
};

static bool valid(const orc_params* p) {
    if (!p || p->k < 3 || p->k > 127 || (p->k % 2) == 0) return false;
    if (p->l < 1 || p->l > 32 || p->l > p->k - 1) return false;
    if (p->cutoff < 1 || p->cutoff > 15) return false;
    if (p->graph_count == 0 || (p->graph_count & (p->graph_count - 1))) return false;
    return true;
}

// Graph_Partitioner::process_chunk, live record loop -- src/Graph_Partitioner.cpp:461-597
static void partition(orc_ctx* c, const uint64_t* rec_off, uint64_t n_rec) {
    const uint32_t k = c->p.k, l = c->p.l;
    const uint64_t gmask = c->p.graph_count - 1;
    const uint64_t cap = 2 * (k - 1) - l;  // sup_km1_mer_len_th (:30)
    const unsigned char* all = (const unsigned char*)c->input.data();
    std::vector<uint64_t> H;
    auto emit = [&](uint64_t g, uint64_t src, uint64_t len, bool ld, bool rd) {
        c->recs.push_back(Rec{(uint32_t)g, (uint8_t)len, (uint8_t)(ld | (rd << 1)), src});
    };
    for (uint64_t r = 0; r < n_rec; ++r) {
        const unsigned char* seq = all + rec_off[r];
        const uint64_t n = rec_off[r + 1] - rec_off[r];
        uint64_t last_frag_end = 0;
        while (true) {
            uint64_t frag_beg;
            for (frag_beg = last_frag_end; frag_beg + (k + 1) <= n; ++frag_beg)
                if (is_dna(seq[frag_beg])) break;
            if (frag_beg + (k + 1) > n) break;
            const unsigned char* frag = seq + frag_beg;
            uint64_t frag_len;
            for (frag_len = 1; frag_len < k + 1; ++frag_len)
                if (!is_dna(frag[frag_len])) break;
            if (frag_len < k + 1) { last_frag_end = frag_beg + frag_len; continue; }
            // the fragment runs while bases are DNA; the record is padded past its end (:471)
            uint64_t fl = k + 1;
            while (frag_beg + fl < n && is_dna(frag[fl])) ++fl;
            H.assign(fl - (k - 1) + 1, 0);
            km1_min_hashes(frag, fl, k, l, H.data());
            const uint64_t base = (uint64_t)(frag - all);

            uint64_t cur_off = 0, km1_idx = 0, pos = k - 1;  // frag_len = k - 1 (:512)
            uint64_t cur_g = H[0] & gmask, prev_g = c->p.graph_count, next_g;
            while (pos < fl) {                                // while is_DNA(frag[frag_len])
                const uint64_t len = km1_idx + (k - 1);
                ++km1_idx; ++pos;
                next_g = H[pos - (k - 1)] & gmask;
                if (next_g != cur_g || len == cap) {
                    const uint64_t next_off = cur_off + km1_idx;
                    const bool lj = cur_off > 0;
                    emit(cur_g, base + cur_off - lj, lj + len + 1, lj && prev_g != cur_g, next_g != cur_g);
                    cur_off = next_off;
                    prev_g = cur_g; cur_g = next_g; km1_idx = 0;
                }
            }
            const uint64_t len = pos - cur_off;
            const bool lj = cur_off > 0;
            emit(cur_g, base + cur_off - lj, lj + len, lj && prev_g != cur_g, false);
            last_frag_end = frag_beg + pos;
        }
    }
}

extern "C" {

orc_ctx* orc_create(const orc_params* p) {
    if (!valid(p)) return nullptr;
    return new orc_ctx(*p);
}

void orc_destroy(orc_ctx* c) { delete c; }

static void load(orc_ctx* c, const char* seq, const uint64_t* rec_off, uint64_t n_rec) {
    c->input.assign(seq, rec_off[n_rec]);
    c->recs.clear();
    partition(c, rec_off, n_rec);
    c->rec_g.clear(); c->rec_len.clear(); c->rec_flags.clear(); c->rec_src.clear();
    for (const Rec& r : c->recs) {
        c->rec_g.push_back(r.g); c->rec_len.push_back(r.len);
        c->rec_flags.push_back(r.flags); c->rec_src.push_back(r.src);
    }
}

int orc_partition_only(orc_ctx* c, const char* seq, const uint64_t* rec_off, uint64_t n_rec) {
    if (!c) return 1;
    load(c, seq, rec_off, n_rec);
    return 0;
}

int orc_run(orc_ctx* c, const char* seq, const uint64_t* rec_off, uint64_t n_rec, int n_threads) {
    if (!c) return 1;
    load(c, seq, rec_off, n_rec);
    const uint32_t G = c->p.graph_count;
    std::vector<std::vector<Rec>> bucket(G);
    for (const Rec& r : c->recs) bucket[r.g].push_back(r);
    std::vector<SubOut> outs(G);
    // Subgraphs_Manager::process: larger buckets first, dynamic pull (src/Subgraphs_Manager.cpp:222-255)
    std::vector<uint32_t> order(G);
    for (uint32_t g = 0; g < G; ++g) order[g] = g;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return bucket[a].size() > bucket[b].size(); });
    std::atomic<uint32_t> next{0};
    if (n_threads < 1) n_threads = 1;
    auto work = [&]() {
        Worker w(c->kc, c->p.cutoff);
        while (true) {
            const uint32_t i = next.fetch_add(1);
            if (i >= G) break;
            const uint32_t g = order[i];
            if (bucket[g].empty()) continue;
            w.construct(bucket[g], c->input, outs[g]);
            w.contract(outs[g]);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < n_threads; ++t) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();

    c->vtx_g.clear(); c->vtx_key.clear(); c->vtx_ef.clear(); c->vtx_status.clear();
    c->fasta.clear(); c->lm_text.clear(); c->lm_off.assign(1, 0);
    c->lm_u.clear(); c->lm_v.clear(); c->lm_flags.clear(); c->lm_g.clear();
    c->n_inst = c->n_vert = c->n_iso = c->n_phan = c->n_triv = c->n_icc = c->n_lm = c->n_edges = 0;
    for (uint32_t g = 0; g < G; ++g) {
        SubOut& o = outs[g];
        for (size_t i = 0; i < o.vkeys.size(); ++i) {
            c->vtx_g.push_back(g);
            for (int j = KW - 1; j >= 0; --j) c->vtx_key.push_back(o.vkeys[i].w[j]);   // highest word first
            c->vtx_ef.push_back(o.vstates[i].ef); c->vtx_status.push_back(o.vstates[i].st);
        }
        c->fasta += o.fasta;
        uint64_t off = c->lm_text.size();
        c->lm_text += o.lm_text;
        for (size_t i = 0; i < o.lm_len.size(); ++i) {
            off += o.lm_len[i];
            c->lm_off.push_back(off);
            for (int j = KW - 1; j >= 0; --j) c->lm_u.push_back(o.lm_u[i].w[j]);
            for (int j = KW - 1; j >= 0; --j) c->lm_v.push_back(o.lm_v[i].w[j]);
            c->lm_flags.push_back(o.lm_flags[i]);
            c->lm_g.push_back(g);
        }
        c->n_inst += o.n_inst; c->n_vert += o.vkeys.size(); c->n_iso += o.n_isolated;
        c->n_phan += o.n_phantom; c->n_triv += o.n_trivial; c->n_icc += o.n_icc;
        c->n_lm += o.n_lmtig; c->n_edges += o.n_edges;
        o = SubOut();
    }
    return 0;
}

int orc_get(orc_ctx* c, orc_result* o) {
    if (!c || !o) return 1;
    o->n_records = c->recs.size();
    o->n_instances = c->n_inst; o->n_vertices = c->n_vert; o->n_isolated = c->n_iso;
    o->n_phantom = c->n_phan; o->n_trivial = c->n_triv; o->n_icc = c->n_icc; o->n_lmtig = c->n_lm;
    o->n_edges = c->n_edges;
    o->rec_g = c->rec_g.data(); o->rec_len = c->rec_len.data(); o->rec_flags = c->rec_flags.data();
    o->rec_src = c->rec_src.data();
    o->vtx_g = c->vtx_g.data(); o->vtx_key = c->vtx_key.data(); o->vtx_ef = c->vtx_ef.data();
    o->vtx_status = c->vtx_status.data();
    o->fasta_bytes = c->fasta.size(); o->fasta = c->fasta.data();
    o->lm_text = c->lm_text.data(); o->lm_off = c->lm_off.data(); o->lm_u = c->lm_u.data();
    o->lm_v = c->lm_v.data(); o->lm_flags = c->lm_flags.data(); o->lm_g = c->lm_g.data();
    return 0;
}

int orc_record_labels(orc_ctx* c, char* out, uint64_t cap) {
    uint64_t w = 0;
    for (const Rec& r : c->recs) {
        if (w + r.len > cap) return 1;
        for (uint32_t i = 0; i < r.len; ++i) out[w++] = CHR[map_base((unsigned char)c->input[r.src + i])];
    }
    return 0;
}

uint64_t orc_wyhash8(uint64_t x) { return wyhash8(x); }

uint64_t orc_lmer_hash(uint64_t lmer, uint32_t l) {
    uint64_t rc = 0;
    for (uint32_t i = 0; i < l; ++i) rc = (rc << 2) | (3 - ((lmer >> (2 * i)) & 3));
    return lmer_hash(lmer, rc);
}

int orc_km1_min_hashes(const char* s, uint64_t n, uint32_t k, uint32_t l, uint64_t* out) {
    if (k < 3 || l < 1 || l > k - 1 || l > 32 || n < k - 1) return 1;
    km1_min_hashes((const unsigned char*)s, n, k, l, out);
    return 0;
}

void orc_state_update(uint32_t* ef, uint8_t* status, int front, int back, int s0, int s1) {
    State s; s.ef = *ef; s.st = *status;
    update_edges(s, (uint8_t)front, (uint8_t)back);
    if (s0 != UNSPEC) mark_disc(s, (Side)s0);
    if (s1 != UNSPEC) mark_disc(s, (Side)s1);
    *ef = s.ef; *status = s.st;
}

int orc_edge_at(uint32_t ef, int side, uint32_t f_th) { return edge_at(ef, (Side)side, f_th); }

/* Comparison helper for large parity cases (not part of the restated algorithm):
 * a 64-bit hash of each text span [off[i], off[i] + len[i]), length included. */
void orc_hash_spans(const char* text, const uint64_t* off, const uint64_t* len, uint64_t n, uint64_t* out) {
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t h = 0x9E3779B97F4A7C15ull ^ (len[i] * 0xC2B2AE3D27D4EB4Full);
        const unsigned char* p = (const unsigned char*)text + off[i];
        for (uint64_t j = 0; j < len[i]; ++j) {
            h = (h ^ p[j]) * 0x100000001B3ull;
            h ^= h >> 29;
        }
        h ^= h >> 33; h *= 0xFF51AFD7ED558CCDull; h ^= h >> 33;
        out[i] = h;
    }
}

}  // extern "C"
