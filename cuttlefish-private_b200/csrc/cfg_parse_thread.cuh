// cfg_parse_thread.cuh -- what one thread of the device text parser (cfg_parse.cu) does
// with its 16 bytes, as __host__ __device__ code: the kernels run these steps on the
// GPU, and a host harness in the tests runs the very same steps over every (chunk,
// thread) of a text to check them on a CPU.
//
// Bytes have five classes (newline, '>', a base letter, '\r', other); a finite-state
// machine over the classes (the line structure of FASTA or FASTQ) gives each byte an
// emission: skipped, a base, or a break (a non-ACGT character, a record boundary).
//
// Most 16-byte groups of a real file lie inside one line -- bases of a sequence line,
// quality letters, a header -- where the state loops on every byte.  For those the
// counts, the transfer function and the 2-bit codes come from word-wise byte compares
// (SWAR) instead of a walk of the FSM byte by byte; every other group takes the walk.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define CFG_PHD __host__ __device__ __forceinline__
#else
#define CFG_PHD inline
#endif

namespace cfg {
namespace parse {

constexpr uint32_t CHUNK = 4096, TPB = 256, BPT = CHUNK / TPB;   // bytes per thread: 16
enum : uint32_t { C_NL = 0, C_GT = 1, C_BASE = 2, C_CR = 3, C_OTHER = 4, NCLASS = 5 };
enum : uint32_t { E_SKIP = 0, E_BASE = 1, E_BREAK = 2 };

// The tables of an FSM of at most 5 states packed into registers: entry (class c, state s)
// at index i = 5 c + s, its next state in 3 bits (bits 3i.. of nx_lo for i < 21, of nx_hi
// above) and its emission in 2 bits of em.  A lookup is a few shifts on values every
// thread holds, where an indexed table (in the kernel's parameters or in memory) would
// serialise the warp's lanes over their distinct (state, class) pairs.
struct FsmBits {
    unsigned long long nx_lo, nx_hi, em;
    // class c's whole next-state map as a transfer function (3 bits per state): bits 15c..
    // of cf_lo for c < 4, cf_hi for c = 4; idem bit c: that map is idempotent (a run of
    // class-c bytes acts as one)
    unsigned long long cf_lo;
    uint32_t cf_hi, idem;
    uint32_t n, start;
    // word-wise groups: loop_mask bit s -- state s stays s on a base and on an other byte;
    // gt_other -- '>' has the next states and emissions of an other byte in every state
    // (it is then no delimiter); bo_idem -- bases and other bytes have one class map, and
    // it is idempotent (a group of them composes to that map)
    uint32_t loop_mask, gt_other, bo_idem;
};

CFG_PHD uint32_t fsm_next(const FsmBits& f, uint32_t st, uint32_t cl) {
    const uint32_t i = 5 * cl + st;
    return i < 21 ? (uint32_t)(f.nx_lo >> (3 * i)) & 7u : (uint32_t)(f.nx_hi >> (3 * (i - 21))) & 7u;
}
CFG_PHD uint32_t fsm_emit(const FsmBits& f, uint32_t st, uint32_t cl) {
    return (uint32_t)(f.em >> (2 * (5 * cl + st))) & 3u;
}
CFG_PHD uint32_t class_fn(const FsmBits& f, uint32_t cl) {
    return cl < 4 ? (uint32_t)(f.cf_lo >> (15 * cl)) & 0x7FFFu : f.cf_hi;
}
CFG_PHD uint32_t byte_class(uint32_t c) {
    if (c == '\n') return C_NL;
    if (c == '>') return C_GT;
    if (c == '\r') return C_CR;
    const uint32_t u = c & 0xDF;
    return (u == 'A' || u == 'C' || u == 'G' || u == 'T') ? C_BASE : C_OTHER;
}
CFG_PHD uint32_t base_code(uint32_t c) {   // A0 C1 G2 T3 (case-insensitive)
    const uint32_t u = c & 0xDF;
    return u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : 3;
}
CFG_PHD uint32_t f_at(uint32_t f, uint32_t s) { return (f >> (3 * s)) & 7; }
CFG_PHD uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }
// first f, then g
CFG_PHD uint32_t compose(uint32_t f, uint32_t g, uint32_t n) {
    uint32_t h = 0;
    for (uint32_t s = 0; s < n; ++s) h |= f_at(g, f_at(f, s)) << (3 * s);
    return h;
}
CFG_PHD uint32_t identity(uint32_t n) {
    uint32_t h = 0;
    for (uint32_t s = 0; s < n; ++s) h |= s << (3 * s);
    return h;
}

CFG_PHD uint32_t popc32(uint32_t x) {
#ifdef __CUDA_ARCH__
    return (uint32_t)__popc(x);
#else
    return (uint32_t)__builtin_popcount(x);
#endif
}

// A thread's 16 bytes as four little-endian words: byte i is bits 8(i%4).. of w[i/4].
struct Group { uint32_t w[4]; };

CFG_PHD uint32_t byte_at(const Group& g, uint32_t i) { return (g.w[i >> 2] >> (8 * (i & 3))) & 0xFFu; }

// 0x80 in every byte of x that equals the byte value b, 0 in every other byte (exact:
// no byte's sum carries into the next)
CFG_PHD uint32_t eq_bytes(uint32_t x, uint32_t b) {
    const uint32_t y = x ^ (b * 0x01010101u);
    return ~(((y & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | y) & 0x80808080u;
}

// Whether the group holds a newline, a '\r' or -- unless it acts as an other byte -- a '>'.
CFG_PHD bool has_delimiter(const FsmBits& f, const Group& g) {
    uint32_t m = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        m |= eq_bytes(g.w[i], '\n') | eq_bytes(g.w[i], '\r');
        if (!f.gt_other) m |= eq_bytes(g.w[i], '>');
    }
    return m != 0;
}

// Base letters (ACGT, either case) among the group's bytes.
CFG_PHD uint32_t count_acgt(const Group& g) {
    uint32_t n = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t u = g.w[i] & 0xDFDFDFDFu;
        n += popc32(eq_bytes(u, 'A') | eq_bytes(u, 'C') | eq_bytes(u, 'G') | eq_bytes(u, 'T'));
    }
    return n;
}

// The transfer function of nb bytes (nb <= 16): the class maps composed in byte order, a
// run of one idempotent class composed once; a full group without delimiters is one
// composition when bases and other bytes share an idempotent map.
CFG_PHD uint32_t thread_transfer(const FsmBits& f, const Group& g, uint32_t nb) {
    if (nb == BPT && f.bo_idem && !has_delimiter(f, g)) return class_fn(f, C_BASE);
    uint32_t fn = identity(f.n), prev = NCLASS;
#pragma unroll
    for (uint32_t i = 0; i < BPT; ++i) {
        if (i >= nb) break;
        const uint32_t cl = byte_class(byte_at(g, i));
        if (cl != prev || !((f.idem >> cl) & 1)) fn = compose(fn, class_fn(f, cl), f.n);
        prev = cl;
    }
    return fn;
}

// Bases and breaks the group emits from state st.
CFG_PHD void thread_counts(const FsmBits& f, uint32_t st, const Group& g, uint32_t nbytes, uint32_t& nb, uint32_t& nk) {
    if (nbytes == BPT && ((f.loop_mask >> st) & 1) && !has_delimiter(f, g)) {
        // the state stays st on every byte: bases and other bytes emit one kind each
        const uint32_t eb = fsm_emit(f, st, C_BASE), eo = fsm_emit(f, st, C_OTHER);
        const uint32_t na = eb == eo ? BPT : count_acgt(g), no = BPT - na;
        nb = (eb == E_BASE ? na : 0u) + (eo == E_BASE ? no : 0u);
        nk = (eb == E_BREAK ? na : 0u) + (eo == E_BREAK ? no : 0u);
        return;
    }
    nb = nk = 0;
#pragma unroll
    for (uint32_t i = 0; i < BPT; ++i) {
        if (i >= nbytes) break;
        const uint32_t cl = byte_class(byte_at(g, i));
        const uint32_t e = fsm_emit(f, st, cl);
        nb += e == E_BASE; nk += e == E_BREAK;
        st = fsm_next(f, st, cl);
    }
}

// The rank (bases before it) of each break the group emits: r bases and kk breaks precede
// the group's first byte.
CFG_PHD void thread_breaks(const FsmBits& f, uint32_t st, const Group& g, uint32_t nbytes, unsigned long long r,
                           unsigned long long kk, unsigned long long* brk_rank) {
#pragma unroll
    for (uint32_t i = 0; i < BPT; ++i) {
        if (i >= nbytes) break;
        const uint32_t cl = byte_class(byte_at(g, i));
        const uint32_t e = fsm_emit(f, st, cl);
        if (e == E_BASE) ++r;
        else if (e == E_BREAK) brk_rank[kk++] = r;
        st = fsm_next(f, st, cl);
    }
}

// 2-bit codes (A0 C1 G2 T3) of 16 base letters of either case, byte 0's in bits 31:30:
// ((c >> 1) ^ (c >> 2)) & 3 is a letter's code (A 0x41, C 0x43, G 0x47, T 0x54 and
// their lower-case forms), and the masks keep each byte's code inside its byte.
CFG_PHD uint32_t pack16(const Group& g) {
    uint32_t p = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const uint32_t c = ((g.w[i] >> 1) ^ (g.w[i] >> 2)) & 0x03030303u;
        const uint32_t q = ((c & 3u) << 6) | (((c >> 8) & 3u) << 4) | (((c >> 16) & 3u) << 2) | ((c >> 24) & 3u);
        p = (p << 8) | q;
    }
    return p;
}

// Where the packed stream wants base i of fragment kk: out[kk] + (bases before it in the
// fragment); ~0 for a dropped fragment.
struct FragPos {
    unsigned long long out, first;   // the fragment's output start, the rank of its first base
};
CFG_PHD FragPos frag_pos(const unsigned long long* frag_out, const unsigned long long* brk_rank, unsigned long long kk) {
    return FragPos{frag_out[kk], kk ? brk_rank[kk - 1] : 0ull};
}

// The group's bases into the packed stream (MSB-first, 32 per word, every word zero
// before the pass): r bases and kk breaks precede the group; nb and nk are the group's
// own counts.  or64(word pointer, bits) merges bits into a word (an atomic on the GPU:
// a word's bases may come from two threads).
template <class Or64>
CFG_PHD void thread_pack(const FsmBits& f, uint32_t st, const Group& g, uint32_t nbytes, unsigned long long r,
                         unsigned long long kk, uint32_t nb, uint32_t nk, const unsigned long long* frag_out,
                         const unsigned long long* brk_rank, uint64_t* packed, Or64 or64) {
    if (nb == 0) return;
    FragPos fp = frag_pos(frag_out, brk_rank, kk);
    if (nb == BPT && nk == 0) {   // 16 bases of one fragment, in a row
        if (fp.out == ~0ull) return;
        const unsigned long long q = fp.out + (r - fp.first);
        const uint64_t s = (uint64_t)pack16(g) << 32;   // byte 0's base at bits 63:62
        const uint32_t o = (uint32_t)(q & 31);
        or64(packed + (q >> 5), s >> (2 * o));
        if (o > 16) or64(packed + (q >> 5) + 1, s << (64 - 2 * o));
        return;
    }
    uint64_t word = ~0ull, acc = 0;
#pragma unroll
    for (uint32_t i = 0; i < BPT; ++i) {
        if (i >= nbytes) break;
        const uint32_t ch = byte_at(g, i), cl = byte_class(ch);
        const uint32_t e = fsm_emit(f, st, cl);
        if (e == E_BASE) {
            if (fp.out != ~0ull) {
                const unsigned long long q = fp.out + (r - fp.first);
                const uint64_t w = q >> 5;
                if (w != word) {
                    if (word != ~0ull) or64(packed + word, acc);
                    word = w; acc = 0;
                }
                acc |= (uint64_t)base_code(ch) << (62 - 2 * (q & 31));
            }
            ++r;
        } else if (e == E_BREAK) {
            fp = frag_pos(frag_out, brk_rank, ++kk);
        }
        st = fsm_next(f, st, cl);
    }
    if (word != ~0ull) or64(packed + word, acc);
}

// A thread's exclusive prefix of bases (low 16 bits) and breaks (high 16 bits) within its
// chunk; the 255 threads before it hold at most 4080 bytes.
CFG_PHD uint32_t pre_pack(uint32_t eb, uint32_t ek) { return eb | (ek << 16); }
CFG_PHD uint32_t pre_bases(uint32_t p) { return p & 0xFFFFu; }
CFG_PHD uint32_t pre_breaks(uint32_t p) { return p >> 16; }

// After pass D: bases and breaks before thread t's bytes (r, kk) and its own (nb, nk),
// from pass C's per-thread prefixes (the next thread's, or the chunk's totals for the
// last thread of a chunk); chunk_b / chunk_k hold the chunks' exclusive prefixes, with
// the totals at index n_chunks.
struct ThreadSpan { unsigned long long r, kk; uint32_t nb, nk; };
CFG_PHD ThreadSpan thread_span(const uint32_t* thread_pre, const unsigned long long* chunk_b,
                               const unsigned long long* chunk_k, uint64_t c, uint32_t t) {
    const uint64_t i = c * TPB + t;
    const uint32_t p = thread_pre[i];
    const unsigned long long cb = chunk_b[c], ck = chunk_k[c];
    uint32_t eb1, ek1;
    if (t + 1 < TPB) {
        const uint32_t q = thread_pre[i + 1];
        eb1 = pre_bases(q); ek1 = pre_breaks(q);
    } else {
        eb1 = (uint32_t)(chunk_b[c + 1] - cb); ek1 = (uint32_t)(chunk_k[c + 1] - ck);
    }
    return ThreadSpan{cb + pre_bases(p), ck + pre_breaks(p), eb1 - pre_bases(p), ek1 - pre_breaks(p)};
}

// ---------------------------------------------------------------------------------------
// The machines (host): their tables, and the packed form the kernels read.

// Up to 8 states; a transfer function packs the image of each state in 3 bits.
struct Fsm {
    uint8_t next[8][NCLASS];
    uint8_t emit[8][NCLASS];
    uint32_t n, start;
};

inline FsmBits pack_fsm(const Fsm& m) {
    FsmBits b{};
    b.n = m.n; b.start = m.start;
    for (uint32_t c = 0; c < NCLASS; ++c) {
        uint32_t F = 0;
        bool idem = true;
        for (uint32_t st = 0; st < m.n; ++st) {
            const uint32_t i = 5 * c + st;
            if (i < 21) b.nx_lo |= (unsigned long long)m.next[st][c] << (3 * i);
            else b.nx_hi |= (unsigned long long)m.next[st][c] << (3 * (i - 21));
            b.em |= (unsigned long long)m.emit[st][c] << (2 * i);
            F |= (uint32_t)m.next[st][c] << (3 * st);
            idem = idem && m.next[m.next[st][c]][c] == m.next[st][c];
        }
        if (c < 4) b.cf_lo |= (unsigned long long)F << (15 * c); else b.cf_hi = F;
        if (idem) b.idem |= 1u << c;
    }
    // word-wise groups (cfg_parse_thread.cuh): states that loop on bases and other bytes,
    // '>' as an other byte, and one idempotent map for bases and other bytes
    b.gt_other = 1;
    b.bo_idem = 1;
    for (uint32_t st = 0; st < m.n; ++st) {
        if (m.next[st][C_BASE] == st && m.next[st][C_OTHER] == st) b.loop_mask |= 1u << st;
        if (m.next[st][C_GT] != m.next[st][C_OTHER] || m.emit[st][C_GT] != m.emit[st][C_OTHER]) b.gt_other = 0;
        if (m.next[st][C_BASE] != m.next[st][C_OTHER] || m.next[m.next[st][C_BASE]][C_BASE] != m.next[st][C_BASE])
            b.bo_idem = 0;
    }
    return b;
}

inline Fsm fasta_fsm() {
    // states: 0 line start before any record, 1 inside such a line, 2 header,
    // 3 line start inside a record, 4 sequence line
    Fsm m{};
    m.n = 5; m.start = 0;
    auto set = [&](uint32_t s, uint32_t c, uint32_t nx, uint32_t e) { m.next[s][c] = (uint8_t)nx; m.emit[s][c] = (uint8_t)e; };
    for (uint32_t c = 0; c < NCLASS; ++c) {
        set(0, c, 1, E_SKIP); set(1, c, 1, E_SKIP); set(2, c, 2, E_SKIP);
        set(3, c, 4, E_BREAK); set(4, c, 4, E_BREAK);
    }
    set(0, C_NL, 0, E_SKIP); set(0, C_CR, 0, E_SKIP); set(0, C_GT, 2, E_BREAK);
    set(1, C_NL, 0, E_SKIP);
    set(2, C_NL, 3, E_SKIP);
    set(3, C_NL, 3, E_SKIP); set(3, C_GT, 2, E_BREAK); set(3, C_BASE, 4, E_BASE);
    set(4, C_NL, 3, E_SKIP); set(4, C_BASE, 4, E_BASE);
    return m;
}

inline Fsm fastq_fsm() {
    // states: 0 before a record (blank lines skipped), 1 header line, 2 sequence line,
    // 3 '+' line, 4 quality line
    Fsm m{};
    m.n = 5; m.start = 0;
    auto set = [&](uint32_t s, uint32_t c, uint32_t nx, uint32_t e) { m.next[s][c] = (uint8_t)nx; m.emit[s][c] = (uint8_t)e; };
    for (uint32_t c = 0; c < NCLASS; ++c) {
        set(0, c, 1, E_SKIP); set(1, c, 1, E_SKIP); set(2, c, 2, E_BREAK); set(3, c, 3, E_SKIP); set(4, c, 4, E_SKIP);
    }
    set(0, C_NL, 0, E_SKIP); set(0, C_CR, 0, E_SKIP);
    set(1, C_NL, 2, E_SKIP);
    set(2, C_NL, 3, E_BREAK); set(2, C_BASE, 2, E_BASE);
    set(3, C_NL, 4, E_SKIP);
    set(4, C_NL, 0, E_SKIP);
    return m;
}

}  // namespace parse
}  // namespace cfg
