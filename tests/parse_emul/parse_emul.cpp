// parse_emul.cpp -- the device text parser (cuttlefish-private_b200/csrc/cfg_parse.cu) run
// on a CPU, for the tests.  Every per-thread step is the parser's own code
// (cfg_parse_thread.cuh: transfer functions, counts, break ranks, packing, the per-thread
// spans), run here for every (chunk, thread) in order; the scans the kernels do across a
// CTA (shuffles, shared memory) and across chunks (one-CTA passes) are plain loops, and
// the fragment pass F -- unchanged kernels -- is restated in a few lines.  The tests
// compare its packed stream and fragment table with the host packer's.
//
// Also exported: a self-test of the word-wise steps (SWAR classification, counts,
// transfer functions, 2-bit codes) against the byte-by-byte FSM walk on random groups.
#include "cfg_parse_thread.cuh"

#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

using namespace cfg::parse;

namespace {

Group load_group(const uint8_t* text, uint64_t bytes, uint64_t c, uint32_t t) {
    const uint64_t p = c * CHUNK + (uint64_t)t * BPT;
    Group g{};
    for (int j = 0; j < 4; ++j) {
        uint32_t x = 0;
        for (int i = 0; i < 4; ++i)
            if (p + 4 * j + i < bytes) x |= (uint32_t)text[p + 4 * j + i] << (8 * i);
        g.w[j] = x;
    }
    return g;
}

uint32_t bytes_of_thread(uint64_t bytes, uint64_t c, uint32_t t) {
    const uint64_t p = c * CHUNK + (uint64_t)t * BPT;
    return p >= bytes ? 0 : (uint32_t)umin64(BPT, bytes - p);
}

struct HostOr64 {
    void operator()(uint64_t* w, uint64_t bits) const { *w |= bits; }
};

// the byte-by-byte walk: counts, final state and transfer function of nb bytes
void walk(const FsmBits& f, uint32_t st, const Group& g, uint32_t nbytes, uint32_t& nb, uint32_t& nk, uint32_t& fn) {
    nb = nk = 0;
    fn = identity(f.n);
    for (uint32_t i = 0; i < nbytes; ++i) {
        const uint32_t cl = byte_class(byte_at(g, i));
        const uint32_t e = fsm_emit(f, st, cl);
        nb += e == E_BASE; nk += e == E_BREAK;
        st = fsm_next(f, st, cl);
        fn = compose(fn, class_fn(f, cl), f.n);
    }
}

}  // namespace

extern "C" {

// Parses `bytes` of text as the device does; on success *words (n_bases / 32 rounded up,
// plus 4 zero words), *frag_off and *frag_len are malloc'd (free with parse_emul_free).
int parse_emul(const uint8_t* text, uint64_t bytes, int fastq, uint32_t k, uint64_t** words, uint64_t* n_bases,
               uint64_t** frag_off, uint32_t** frag_len, uint64_t* n_frags) {
    const FsmBits f = pack_fsm(fastq ? fastq_fsm() : fasta_fsm());
    const uint64_t nc = (bytes + CHUNK - 1) / CHUNK;
    std::vector<uint32_t> chunk_f(nc + 1), thread_pre(nc * TPB + 1);
    std::vector<uint16_t> thread_f(nc * TPB + 1);
    std::vector<unsigned long long> chunk_b(nc + 1), chunk_k(nc + 1);
    // A: every thread's transfer function; the chunk's exclusive prefix per thread
    for (uint64_t c = 0; c < nc; ++c) {
        uint32_t ex = identity(f.n);
        for (uint32_t t = 0; t < TPB; ++t) {
            const uint32_t fn = thread_transfer(f, load_group(text, bytes, c, t), bytes_of_thread(bytes, c, t));
            thread_f[c * TPB + t] = (uint16_t)ex;
            ex = compose(ex, fn, f.n);
        }
        chunk_f[c] = ex;
    }
    // B: each chunk's start state
    uint32_t st = f.start;
    for (uint64_t c = 0; c < nc; ++c) { const uint32_t tf = chunk_f[c]; chunk_f[c] = st; st = f_at(tf, st); }
    // C: counts, every thread's exclusive prefix within its chunk
    for (uint64_t c = 0; c < nc; ++c) {
        uint32_t eb = 0, ek = 0;
        for (uint32_t t = 0; t < TPB; ++t) {
            uint32_t nb, nk;
            thread_counts(f, f_at(thread_f[c * TPB + t], chunk_f[c]), load_group(text, bytes, c, t),
                          bytes_of_thread(bytes, c, t), nb, nk);
            thread_pre[c * TPB + t] = pre_pack(eb, ek);
            eb += nb; ek += nk;
        }
        chunk_b[c] = eb; chunk_k[c] = ek;
    }
    // D: the chunks' exclusive prefixes, totals at nc
    unsigned long long rb = 0, rk = 0;
    for (uint64_t c = 0; c < nc; ++c) {
        const unsigned long long x = chunk_b[c], y = chunk_k[c];
        chunk_b[c] = rb; chunk_k[c] = rk; rb += x; rk += y;
    }
    chunk_b[nc] = rb; chunk_k[nc] = rk;
    // E: break ranks
    const uint64_t NB = rk;
    std::vector<unsigned long long> brk_rank(NB + 1), frag_out(NB + 1);
    for (uint64_t c = 0; c < nc; ++c)
        for (uint32_t t = 0; t < TPB; ++t) {
            const ThreadSpan sp = thread_span(thread_pre.data(), chunk_b.data(), chunk_k.data(), c, t);
            if (sp.nk == 0) continue;
            thread_breaks(f, f_at(thread_f[c * TPB + t], chunk_f[c]), load_group(text, bytes, c, t),
                          bytes_of_thread(bytes, c, t), sp.r, sp.kk, brk_rank.data());
        }
    brk_rank[NB] = rb;
    // F: fragments of at least k+1 bases, their output starts
    std::vector<uint64_t> fo;
    std::vector<uint32_t> fl;
    unsigned long long at = 0;
    for (uint64_t i = 0; i <= NB; ++i) {
        const unsigned long long L = brk_rank[i] - (i ? brk_rank[i - 1] : 0ull);
        if (L >= k + 1) { frag_out[i] = at; fo.push_back(at); fl.push_back((uint32_t)L); at += L; }
        else frag_out[i] = ~0ull;
    }
    // G: packing
    const uint64_t nw = (at + 31) / 32 + 4;
    uint64_t* w = (uint64_t*)std::calloc(nw, 8);
    uint64_t* o = (uint64_t*)std::malloc(8 * (fo.size() + 1));
    uint32_t* l = (uint32_t*)std::malloc(4 * (fl.size() + 1));
    if (!w || !o || !l) { std::free(w); std::free(o); std::free(l); return 1; }
    for (uint64_t c = 0; c < nc; ++c)
        for (uint32_t t = 0; t < TPB; ++t) {
            const ThreadSpan sp = thread_span(thread_pre.data(), chunk_b.data(), chunk_k.data(), c, t);
            if (sp.nb == 0) continue;
            thread_pack(f, f_at(thread_f[c * TPB + t], chunk_f[c]), load_group(text, bytes, c, t),
                        bytes_of_thread(bytes, c, t), sp.r, sp.kk, sp.nb, sp.nk, frag_out.data(), brk_rank.data(), w,
                        HostOr64{});
        }
    if (!fo.empty()) { std::memcpy(o, fo.data(), 8 * fo.size()); std::memcpy(l, fl.data(), 4 * fl.size()); }
    *words = w; *n_bases = at; *frag_off = o; *frag_len = l; *n_frags = fo.size();
    return 0;
}

void parse_emul_free(void* p) { std::free(p); }

// The word-wise flags of a machine: loop_mask, gt_other, bo_idem.
void parse_emul_fsm_flags(int fastq, uint32_t out[3]) {
    const FsmBits f = pack_fsm(fastq ? fastq_fsm() : fasta_fsm());
    out[0] = f.loop_mask; out[1] = f.gt_other; out[2] = f.bo_idem;
}

// Random groups (bytes drawn mostly from letters, quality and delimiter characters): the
// word-wise counts and transfer functions against the byte-by-byte walk in every state of
// both machines, and the 2-bit codes of all-letter groups against base_code.  Returns
// the number of mismatches.
uint64_t parse_emul_selftest(uint64_t seed, uint64_t iters) {
    static const char alpha[] = "ACGTacgtNnIII#+@>>\n\r\n ";
    std::mt19937_64 rng(seed);
    const FsmBits fs[2] = {pack_fsm(fasta_fsm()), pack_fsm(fastq_fsm())};
    uint64_t bad = 0;
    for (uint64_t it = 0; it < iters; ++it) {
        Group g{};
        const uint64_t mode = rng() % 4;
        for (int i = 0; i < 16; ++i) {
            uint32_t b;
            if (mode == 0) b = (uint32_t)(rng() & 0xFF);                           // any byte
            else if (mode == 1) b = (uint32_t)"ACGTacgt"[rng() % 8];                // all letters
            else if (mode == 2) b = (uint32_t)alpha[rng() % (sizeof(alpha) - 1)];   // mixed
            else b = (uint32_t)"ACGTIIII>N"[rng() % 10];                            // no newline
            g.w[i >> 2] |= b << (8 * (i & 3));
        }
        const uint32_t nbytes = (rng() % 8 == 0) ? (uint32_t)(rng() % 17) : BPT;
        for (const FsmBits& f : fs) {
            for (uint32_t st = 0; st < f.n; ++st) {
                uint32_t nb, nk, wb, wk, wf;
                thread_counts(f, st, g, nbytes, nb, nk);
                walk(f, st, g, nbytes, wb, wk, wf);
                bad += nb != wb || nk != wk;
            }
            uint32_t wb, wk, wf;
            walk(f, f.start, g, nbytes, wb, wk, wf);
            bad += thread_transfer(f, g, nbytes) != wf;
        }
        if (mode == 1) {
            uint32_t p = 0;
            for (uint32_t i = 0; i < 16; ++i) p = (p << 2) | base_code(byte_at(g, i));
            bad += pack16(g) != p;
        }
    }
    return bad;
}

}  // extern "C"
