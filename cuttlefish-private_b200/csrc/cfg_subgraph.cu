// cfg_subgraph.cu -- K2 + K3: per-subgraph vertex table and local unitig walk.
//
// One subgraph is owned by one CTA, or by a thread-block cluster of up to 8
// CTAs whose shared memories together hold the subgraph's open-addressing
// table (slot s lives in CTA s / per, reached through distributed shared
// memory).  Subgraphs too large for a cluster use a global-memory arena with
// the same code.  Per vertex the table holds the canonical k-mer, one 64-bit
// state word -- the packed 4-bit edge frequencies of State_Config<false>
// (include/State_Config.hpp:24-268) in the low half and the stream position of
// the vertex's first occurrence in the high half -- and a meta word
// (discontinuity flags, then the walk's bookkeeping).
//
// Build (Subgraph::construct, src/Subgraph.cpp:43-108): every thread of the
// CTA/cluster takes weak super k-mers, rolls their k-mers and applies
// HT_Router::update (include/Subgraph.hpp:546-560) as one CAS on the state word
// (saturated counts and an unchanged first occurrence need no CAS).  The
// self-loop rule (:82-83) needs only the previous k-mer of the same super k-mer.
//
// Walk (Subgraph::contract / extract_maximal_unitig / walk_unitig,
// src/Subgraph.cpp:183-271, include/Subgraph.hpp:414-543): a step v -(side s)-> u
// is taken iff s holds one passing edge, u != v, and u's entrance side holds at
// most one.  That relation is symmetric, so the reference's sequential walk from
// any seed returns the whole maximal path whatever the seed order, except in one
// case: a homopolymer vertex b^k whose back side holds only its own self-loop and
// whose front side holds at most one edge.  Seeded directly, the reference
// records it as a one-vertex cycle; reached from its predecessor, it ends that
// predecessor's unitig.  The reference seeds in table-insertion order (first
// occurrence), so the kernel compares first-occurrence positions to decide, and
// orients each lm-tig by its first-inserted vertex exactly as the reference does.
// Paths are walked from both ends in parallel; the end with the smaller slot emits.
#include <cooperative_groups.h>

#include "cfg_device.cuh"
#include "cfg_internal.h"

namespace cg = cooperative_groups;

namespace cfg {

namespace {

constexpr uint32_t NONE = 0xffffffffu;
constexpr uint64_t EMPTY = ~0ull;
constexpr uint64_t BUSY = ~1ull;   // a three- or four-word key's highest word while the others are written
constexpr uint64_t ST_INIT = 0xffffffff00000000ull;   // a new slot's state: no edges, first occurrence "none"
// walk termination kinds (Walk_Termination, include/Subgraph.hpp:362-369)
constexpr uint32_t T_OK = 0, T_BRANCHED = 1, T_CROSSED = 2, T_DEAD = 3, T_EXIT = 4;
// meta layout: bits 0-2 visited / disc front / disc back; 3 isolated; 4-17 the front side
// and 18-31 the back side.  A side is 1 | u << 1 | s_in << 13 when its walk step leads to
// slot u, entered by side s_in (one-CTA tables of at most LINK_SLOTS slots: the walks
// follow these links instead of looking the neighbour up again), else its termination
// kind << 1 (T_OK, 0, for an unlinked side that continues).
constexpr uint32_t M_ISO = 8u;
constexpr uint32_t LINK_SLOTS = 4096;
enum { LOCAL = 0, CLUSTER = 1, GLOBAL = 2 };

__device__ __forceinline__ uint32_t side_field(uint32_t meta, int side) { return (meta >> (side == FRONT ? 4 : 18)) & 0x3FFFu; }
__device__ __forceinline__ uint32_t side_bits(uint32_t field, int side) { return field << (side == FRONT ? 4 : 18); }
__device__ __forceinline__ uint32_t term_of(uint32_t meta, int side) {
    const uint32_t f = side_field(meta, side);
    return (f & 1) ? T_OK : f >> 1;
}
__device__ __forceinline__ uint32_t compb(uint32_t b) { return b < 4 ? 3 - b : b; }
__device__ __forceinline__ uint32_t st_ef(uint64_t st) { return (uint32_t)st; }
__device__ __forceinline__ uint32_t st_ins(uint64_t st) { return (uint32_t)(st >> 32); }

// Memory-space accessors.  LOCAL and CLUSTER address a slot by a 32-bit shared
// address (CLUSTER: mapped into the owning CTA with mapa); GLOBAL by a pointer.
// Explicit state spaces keep table traffic on the shared-memory pipes.
template <int MODE> struct Mem;
template <> struct Mem<LOCAL> {
    typedef uint32_t A;
    // volatile: these loads also serve waits on other threads' stores (a weak load may be hoisted)
    static __device__ __forceinline__ uint64_t ld64(A a) { uint64_t v; asm volatile("ld.volatile.shared.u64 %0, [%1];" : "=l"(v) : "r"(a) : "memory"); return v; }
    static __device__ __forceinline__ uint32_t ld32(A a) { uint32_t v; asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory"); return v; }
    static __device__ __forceinline__ void st64(A a, uint64_t v) { asm volatile("st.volatile.shared.u64 [%0], %1;" :: "r"(a), "l"(v) : "memory"); }
    static __device__ __forceinline__ void st32(A a, uint32_t v) { asm volatile("st.volatile.shared.u32 [%0], %1;" :: "r"(a), "r"(v) : "memory"); }
    static __device__ __forceinline__ uint64_t cas64(A a, uint64_t c, uint64_t v) { uint64_t o; asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;" : "=l"(o) : "r"(a), "l"(c), "l"(v) : "memory"); return o; }
    static __device__ __forceinline__ uint64_t exch64(A a, uint64_t v) { uint64_t o; asm volatile("atom.shared.exch.b64 %0, [%1], %2;" : "=l"(o) : "r"(a), "l"(v) : "memory"); return o; }
    static __device__ __forceinline__ void or32(A a, uint32_t v) { asm volatile("red.shared.or.b32 [%0], %1;" :: "r"(a), "r"(v) : "memory"); }
    static __device__ __forceinline__ void fence() { __threadfence_block(); }
    static __device__ __forceinline__ void ld2(A a, uint64_t& x, uint64_t& y) { asm volatile("ld.volatile.shared.v2.u64 {%0, %1}, [%2];" : "=l"(x), "=l"(y) : "r"(a) : "memory"); }
    // 16-byte compare-and-swap of {x, y} at a (16-byte aligned); returns the old pair in ox, oy
    static __device__ __forceinline__ void cas128(A a, uint64_t cx, uint64_t cy, uint64_t nx, uint64_t ny, uint64_t& ox, uint64_t& oy) {
        asm volatile("{\n\t.reg .b128 d, c, n;\n\tmov.b128 c, {%2, %3};\n\tmov.b128 n, {%4, %5};\n\t"
                     "atom.shared.cas.b128 d, [%6], c, n;\n\tmov.b128 {%0, %1}, d;\n\t}"
                     : "=l"(ox), "=l"(oy) : "l"(cx), "l"(cy), "l"(nx), "l"(ny), "r"(a) : "memory");
    }
};
template <> struct Mem<CLUSTER> {
    typedef uint32_t A;
    static __device__ __forceinline__ uint64_t ld64(A a) { uint64_t v; asm volatile("ld.relaxed.cluster.shared::cluster.u64 %0, [%1];" : "=l"(v) : "r"(a) : "memory"); return v; }
    static __device__ __forceinline__ uint32_t ld32(A a) { uint32_t v; asm volatile("ld.relaxed.cluster.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory"); return v; }
    static __device__ __forceinline__ void st64(A a, uint64_t v) { asm volatile("st.relaxed.cluster.shared::cluster.u64 [%0], %1;" :: "r"(a), "l"(v) : "memory"); }
    static __device__ __forceinline__ void st32(A a, uint32_t v) { asm volatile("st.relaxed.cluster.shared::cluster.u32 [%0], %1;" :: "r"(a), "r"(v) : "memory"); }
    static __device__ __forceinline__ uint64_t cas64(A a, uint64_t c, uint64_t v) { uint64_t o; asm volatile("atom.relaxed.cluster.shared::cluster.cas.b64 %0, [%1], %2, %3;" : "=l"(o) : "r"(a), "l"(c), "l"(v) : "memory"); return o; }
    static __device__ __forceinline__ uint64_t exch64(A a, uint64_t v) { uint64_t o; asm volatile("atom.relaxed.cluster.shared::cluster.exch.b64 %0, [%1], %2;" : "=l"(o) : "r"(a), "l"(v) : "memory"); return o; }
    static __device__ __forceinline__ void or32(A a, uint32_t v) { asm volatile("red.relaxed.cluster.shared::cluster.or.b32 [%0], %1;" :: "r"(a), "r"(v) : "memory"); }
    static __device__ __forceinline__ void fence() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }
    static __device__ __forceinline__ void ld2(A a, uint64_t& x, uint64_t& y) { asm volatile("ld.relaxed.cluster.shared::cluster.v2.u64 {%0, %1}, [%2];" : "=l"(x), "=l"(y) : "r"(a) : "memory"); }
    static __device__ __forceinline__ void cas128(A a, uint64_t cx, uint64_t cy, uint64_t nx, uint64_t ny, uint64_t& ox, uint64_t& oy) {
        asm volatile("{\n\t.reg .b128 d, c, n;\n\tmov.b128 c, {%2, %3};\n\tmov.b128 n, {%4, %5};\n\t"
                     "atom.relaxed.cluster.shared::cluster.cas.b128 d, [%6], c, n;\n\tmov.b128 {%0, %1}, d;\n\t}"
                     : "=l"(ox), "=l"(oy) : "l"(cx), "l"(cy), "l"(nx), "l"(ny), "r"(a) : "memory");
    }
};
template <> struct Mem<GLOBAL> {
    typedef uint64_t A;   // generic address of global memory
    static __device__ __forceinline__ uint64_t ld64(A a) { return *(const volatile unsigned long long*)a; }
    static __device__ __forceinline__ uint32_t ld32(A a) { return *(const volatile unsigned int*)a; }
    static __device__ __forceinline__ void st64(A a, uint64_t v) { *(volatile unsigned long long*)a = v; }
    static __device__ __forceinline__ void st32(A a, uint32_t v) { *(volatile unsigned int*)a = v; }
    static __device__ __forceinline__ uint64_t cas64(A a, uint64_t c, uint64_t v) { return atomicCAS((unsigned long long*)a, (unsigned long long)c, (unsigned long long)v); }
    static __device__ __forceinline__ uint64_t exch64(A a, uint64_t v) { return atomicExch((unsigned long long*)a, (unsigned long long)v); }
    static __device__ __forceinline__ void or32(A a, uint32_t v) { atomicOr((unsigned int*)a, v); }
    static __device__ __forceinline__ void fence() { __threadfence(); }
    static __device__ __forceinline__ void ld2(A a, uint64_t& x, uint64_t& y) {
        asm volatile("ld.volatile.v2.u64 {%0, %1}, [%2];" : "=l"(x), "=l"(y) : "l"(a) : "memory");
    }
    static __device__ __forceinline__ void cas128(A a, uint64_t cx, uint64_t cy, uint64_t nx, uint64_t ny, uint64_t& ox, uint64_t& oy) {
        cfg::cas128((unsigned long long*)a, cx, cy, nx, ny, ox, oy);
    }
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t mapa_cluster(uint32_t a, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}

// The table of one subgraph: nranks sub-tables of `per` slots, one per CTA of the
// cluster (one in LOCAL and GLOBAL mode).  A k-mer's sub-table (its owner) and its
// home slot there come from two independent halves of its hash; probing wraps
// inside the sub-table.  The CTAs of a cluster share out the subgraph's weak super
// k-mers and update other CTAs' sub-tables with atomics through DSMEM.
template <int W, int MODE>
struct Tab {
    typedef Mem<MODE> M;
    typedef typename M::A A;
    // this CTA's base addresses: keys, states (ef | ins << 32), meta.  For k <= 31 a slot's
    // key and state are one 16-byte pair (keys + 16 s, st = keys + 8), read by one load.
    A keys, st, meta;
    uint32_t per, shift, pmask; // slots per sub-table; slot s lives in rank s >> shift at index s & pmask
    uint32_t nranks, rank;
    uint32_t* err_flag;         // set when a wait on a key being written exceeds its bound

    __device__ __forceinline__ A addr(A base, uint32_t s, uint32_t bytes) const {
        if constexpr (MODE == CLUSTER) return mapa_cluster(base + (s & pmask) * bytes, s >> shift);
        else return base + (A)s * bytes;
    }
    // a slot's key: 16 bytes for k <= 63 (for k <= 31 with the state word), 32 beyond
    static constexpr uint32_t KB = W <= 2 ? 16 : 32;
    __device__ __forceinline__ A ka(uint32_t s) const { return addr(keys, s, KB); }
    __device__ __forceinline__ A sa(uint32_t s) const { return addr(st, s, W == 1 ? 16 : 8); }
    __device__ __forceinline__ A ma(uint32_t s) const { return addr(meta, s, 4); }

    __device__ __forceinline__ uint64_t ld_st(uint32_t s) const { return M::ld64(sa(s)); }
    __device__ __forceinline__ uint32_t ld_meta(uint32_t s) const { return M::ld32(ma(s)); }
    __device__ __forceinline__ void or_meta(uint32_t s, uint32_t v) const { M::or32(ma(s), v); }

    __device__ __forceinline__ Kmer<W> key(uint32_t s) const {
        const A a = ka(s);
        if constexpr (W == 1) return Kmer<1>{M::ld64(a)};
        else if constexpr (W == 2) return Kmer<2>{M::ld64(a), M::ld64(a + 8)};
        else {
            Kmer<W> x;
#pragma unroll
            for (int j = 0; j < W; ++j) x.w[j] = M::ld64(a + 8 * j);
            return x;
        }
    }
    // owner rank and home index inside the owner's sub-table
    __device__ __forceinline__ void place(const Kmer<W>& x, uint32_t& r, uint32_t& h) const {
        if constexpr (MODE == LOCAL) {
            // one table: a multiplicative hash's top bits pick the home slot
            uint64_t z;
            if constexpr (W == 1) z = x.lo * 0x9E3779B97F4A7C15ull;
            else if constexpr (W == 2) z = (x.lo ^ (x.hi * 0xC2B2AE3D27D4EB4Full)) * 0x9E3779B97F4A7C15ull;
            else z = fold_words(x) * 0x9E3779B97F4A7C15ull;
            r = 0;
            h = (uint32_t)(((z >> 32) * per) >> 32);
        } else {
            const uint64_t z = key_hash(x);
            r = (uint32_t)(((uint64_t)(uint32_t)z * nranks) >> 32);
            h = (uint32_t)(((z >> 32) * per) >> 32);
        }
    }
    // read-only phases, any CTA: the slot of x (NONE if absent) and its state word
    __device__ uint32_t find(const Kmer<W>& x, uint64_t& stv) const {
        uint32_t r, h;
        place(x, r, h);
        const uint32_t b = r * per;
        for (uint32_t p = 0; p < per; ++p) {
            const A a = ka(b + h);
            if constexpr (W == 1) {
                uint64_t top;
                M::ld2(a, top, stv);   // key and state together
                if (top == EMPTY) return NONE;
                if (top == x.lo) return b + h;
            } else if constexpr (W == 2) {
                uint64_t lo, hi;
                M::ld2(a, lo, hi);     // the whole key in one read (the table no longer changes)
                if (hi == EMPTY) return NONE;
                if (hi == x.hi && lo == x.lo) { stv = ld_st(b + h); return b + h; }
            } else {
                const uint64_t top = M::ld64(a + 8 * (W - 1));
                if (top == EMPTY) return NONE;
                if (top == x.hi_word() && low_words_match(a, x)) { stv = ld_st(b + h); return b + h; }
            }
            if (++h == per) h = 0;
        }
        return NONE;
    }
    __device__ __forceinline__ uint32_t find(const Kmer<W>& x) const { uint64_t t; return find(x, t); }
    // words 0 .. W-2 of the key at a equal x's (W >= 2)
    __device__ __forceinline__ bool low_words_match(A a, const Kmer<W>& x) const {
        bool e = true;
#pragma unroll
        for (int j = 0; j < W - 1; ++j) e &= M::ld64(a + 8 * j) == x.word(j);
        return e;
    }
    // build phase: find or insert x in sub-table `owner` starting at its home index h;
    // returns the global slot or NONE.  Other ranks' sub-tables are reached through DSMEM.
    // `seen`: a recent value of the slot's state word, the first expected value of its CAS
    __device__ uint32_t find_or_insert(const Kmer<W>& x, uint32_t owner, uint32_t h, bool& fresh, uint64_t& seen) const {
        fresh = false;
        const uint32_t b = owner * per;
        for (uint32_t p = 0; p < per; ++p) {
            const A a = ka(b + h);
            if constexpr (W == 1) {
                uint64_t cur, stv;
                M::ld2(a, cur, stv);   // key and state together
                if (cur == x.lo) { seen = stv; return b + h; }
                if (cur == EMPTY) {
                    const uint64_t old = M::cas64(a, EMPTY, x.lo);
                    if (old == EMPTY) { fresh = true; seen = ST_INIT; return b + h; }
                    if (old == x.lo) { seen = stv; return b + h; }
                }
            } else if constexpr (W == 2) {
                // two-word key: one 16-byte CAS claims a free slot (both words EMPTY) with the
                // whole key, so no reader waits on half of one.  A plain 16-byte read showing an
                // EMPTY word may have caught a claim in progress (a real key's high word holds
                // k - 32 <= 31 bases and is never EMPTY; its low word may be all ones), so such a
                // slot is read again atomically by the same CAS, which fails on a taken slot.
                uint64_t lo, hi;
                M::ld2(a, lo, hi);
                if (hi == EMPTY || lo == EMPTY) {
                    M::cas128(a, EMPTY, EMPTY, x.lo, x.hi, lo, hi);
                    if (lo == EMPTY && hi == EMPTY) { fresh = true; seen = ST_INIT; return b + h; }
                }
                if (lo == x.lo && hi == x.hi) { seen = M::ld64(sa(b + h)); return b + h; }
            } else {
                // multi-word key: claim the highest word with a 64-bit CAS (EMPTY -> BUSY),
                // write the others, then publish the highest; readers wait (bounded) on BUSY
                const A at = a + 8 * (W - 1);
                uint64_t hi = M::ld64(at);
                if (hi == EMPTY) {
                    hi = M::cas64(at, EMPTY, BUSY);
                    if (hi == EMPTY) {
#pragma unroll
                        for (int j = 0; j < W - 1; ++j) M::st64(a + 8 * j, x.word(j));
                        M::fence();
                        M::exch64(at, x.hi_word());
                        fresh = true;
                        seen = ST_INIT;
                        return b + h;
                    }
                }
                for (uint32_t spin = 0; hi == BUSY; ++spin) {
                    if (spin > (1u << 24)) { atomicOr(err_flag, DERR_CAS_LIMIT); return NONE; }
                    hi = M::ld64(at);
                }
                if (hi == x.hi_word()) {
                    M::fence();
                    if (low_words_match(a, x)) { seen = M::ld64(sa(b + h)); return b + h; }
                }
            }
            if (++h == per) h = 0;
        }
        return NONE;
    }
    // build phase, k <= 31: find or insert x together with its state update.  A free slot
    // is claimed with x's first state by one 16-byte CAS (key and state are one pair; a
    // free slot's state is ST_INIT); a slot holding x gets the state CAS of update_state.
    __device__ uint32_t upsert(const Kmer<W>& x, uint32_t owner, uint32_t h, uint32_t front, uint32_t back, uint32_t pos,
                               uint32_t m, bool& fresh) const {
        static_assert(W == 1, "one-word keys only");
        fresh = false;
        const uint32_t b = owner * per;
        const uint64_t first = (uint64_t)ef_add_m(st_ef(ST_INIT), front, back, m) | ((uint64_t)min(st_ins(ST_INIT), pos) << 32);
        // probe bound: a quarter of a large table (a run that long means the table is
        // close to full: the insert fails and the subgraph is retried with a larger one)
        const uint32_t bound = per > 256 ? per / 4 : per;
        for (uint32_t p = 0; p < bound; ++p) {
            const A a = ka(b + h);
            uint64_t cur, stv;
            M::ld2(a, cur, stv);
            if (cur == EMPTY) {
                M::cas128(a, EMPTY, ST_INIT, x.lo, first, cur, stv);
                if (cur == EMPTY) { fresh = true; return b + h; }
            }
            if (cur == x.lo) { update_state(b + h, front, back, pos, m, stv); return b + h; }
            if (++h == per) h = 0;
        }
        return NONE;
    }
    // state word update: ef gets m instances of the edges, ins the earliest position (one
    // CAS unless unchanged)
    __device__ __forceinline__ void update_state(uint32_t s, uint32_t front, uint32_t back, uint32_t pos, uint32_t m,
                                                 uint64_t cur) const {
        const A a = sa(s);
        for (uint32_t it = 0;; ++it) {
            const uint32_t ef = ef_add_m((uint32_t)cur, front, back, m);
            const uint32_t in = min((uint32_t)(cur >> 32), pos);
            const uint64_t nv = (uint64_t)ef | ((uint64_t)in << 32);
            if (nv == cur) return;
            const uint64_t old = M::cas64(a, cur, nv);
            if (old == cur) return;
            cur = old;
            if (it > (1u << 22)) { atomicOr(err_flag, DERR_CAS_LIMIT); return; }
        }
    }
    __device__ __forceinline__ void mark_disc(uint32_t s, uint32_t disc) const {
        const A a = ma(s);
        if ((M::ld32(a) & disc) != disc) M::or32(a, disc);
    }
};

// Where one subgraph's outputs go: the run's arenas, or its job's regions in a batch.
struct Sink {
    char* fasta; unsigned long long fasta_cap; unsigned long long* fasta_cur;
    char* lm_text; unsigned long long lm_text_cap; unsigned long long* lm_text_cur;
    LmtigOut* lm; unsigned long long lm_cap; unsigned long long* lm_cur;
    unsigned long long* cnt;   // vertices, isolated, phantom, trivial, icc, lmtig
    uint32_t* oflow;           // DERR_OUT_OVERFLOW is raised here
    uint32_t g;                // the subgraph's id within its job
};

__device__ __forceinline__ void sink_for(const SubgraphArgs& a, uint32_t b, Sink& o) {
    if (a.jobs) {
        const uint32_t j = b >> a.g_shift;
        JobOut& J = a.jobs[j];
        unsigned long long* cur = a.job_cur + (size_t)j * JOB_CUR_STRIDE;
        o.fasta = a.fasta + J.fasta_off; o.fasta_cap = J.fasta_cap; o.fasta_cur = cur;
        o.lm_text = a.lm_text + J.lm_text_off; o.lm_text_cap = J.lm_text_cap; o.lm_text_cur = cur + 1;
        o.lm = a.lm + J.lm_off; o.lm_cap = J.lm_cap; o.lm_cur = cur + 2;
        o.cnt = &J.vertices; o.oflow = &J.err; o.g = b & ((1u << a.g_shift) - 1);
    } else {
        const uint32_t st = b & (a.stripes - 1);
        unsigned long long* cur = a.stripe_cur + (size_t)st * JOB_CUR_STRIDE;
        o.fasta = a.fasta + st * a.fasta_cap; o.fasta_cap = a.fasta_cap; o.fasta_cur = cur;
        o.lm_text = a.lm_text + st * a.lm_text_cap; o.lm_text_cap = a.lm_text_cap; o.lm_text_cur = cur + 1;
        o.lm = a.lm + st * a.lm_cap; o.lm_cap = a.lm_cap; o.lm_cur = cur + 2;
        o.cnt = &a.cnt->vertices; o.oflow = a.err; o.g = b;
    }
}

struct Block {   // per-CTA shared bookkeeping (in CLUSTER mode the flags of rank 0 are the cluster's)
    uint32_t inserted, overflow, wl_n, covered;   // covered: vertices of the paths and one-k-mer cycles emitted
    // work-list counters: slots the build claimed, W1's compacted slots (when that list
    // overflowed), path ends W1 found, W3's unvisited vertices
    uint32_t fresh_n, w1_n, end_n, cyc_n;
    uint32_t dd_over;   // the record merge's table filled up
    unsigned long long vertices, isolated, phantom, trivial, icc, lmtig;
    Sink sk;
    unsigned long long rs[3][32];   // reserve_block: per-warp totals (<= 1024 threads), then their offsets
};

constexpr uint32_t FULL = 0xffffffffu;
constexpr uint32_t STEP_BUF = 64;   // bases a path walk keeps for its label (2 bits each)

// Output space reserved for one lane: FASTA bytes, lm-tig records, lm-tig label bytes.
struct Res { unsigned long long fa, lm_idx, lm_off; };

// One atomic per warp and kind instead of one per unitig.  Every lane of the warp
// must call it (the walk loops are uniform over the CTA for that reason).
__device__ __forceinline__ Res reserve_warp(const Sink& sk, unsigned long long fa, uint32_t nlm, unsigned long long lmb) {
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long a = fa, c = lmb;
    uint32_t b = nlm;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long x = __shfl_up_sync(FULL, a, d), z = __shfl_up_sync(FULL, c, d);
        const uint32_t y = __shfl_up_sync(FULL, b, d);
        if (lane >= (uint32_t)d) { a += x; b += y; c += z; }
    }
    const unsigned long long ta = __shfl_sync(FULL, a, 31), tc = __shfl_sync(FULL, c, 31);
    const uint32_t tb = __shfl_sync(FULL, b, 31);
    unsigned long long ba = 0, bb = 0, bc = 0;
    if (lane == 0) {
        if (ta) ba = atomicAdd(sk.fasta_cur, ta);
        if (tb) bb = atomicAdd(sk.lm_cur, (unsigned long long)tb);
        if (tc) bc = atomicAdd(sk.lm_text_cur, tc);
    }
    ba = __shfl_sync(FULL, ba, 0); bb = __shfl_sync(FULL, bb, 0); bc = __shfl_sync(FULL, bc, 0);
    return Res{ba + a - fa, bb + b - nlm, bc + c - lmb};
}

// The same for the whole CTA: one atomic per kind and CTA (the cursors are shared by
// every subgraph of a job, or of an output stripe, that runs at the same time).  Every
// thread of the CTA must call it.
__device__ __forceinline__ Res reserve_block(const Sink& sk, Block& B, unsigned long long fa, uint32_t nlm,
                                             unsigned long long lmb) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    unsigned long long a = fa, c = lmb, b = nlm;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long x = __shfl_up_sync(FULL, a, d), y = __shfl_up_sync(FULL, b, d), z = __shfl_up_sync(FULL, c, d);
        if (lane >= (uint32_t)d) { a += x; b += y; c += z; }
    }
    if (lane == 31) { B.rs[0][wid] = a; B.rs[1][wid] = b; B.rs[2][wid] = c; }
    __syncthreads();
    if (threadIdx.x < 3) {   // thread q: kind q's warp totals into offsets, one atomic
        unsigned long long* r = B.rs[threadIdx.x];
        unsigned long long run = 0;
        for (uint32_t w = 0; w < nw; ++w) { const unsigned long long t = r[w]; r[w] = run; run += t; }
        unsigned long long* cur = threadIdx.x == 0 ? sk.fasta_cur : threadIdx.x == 1 ? sk.lm_cur : sk.lm_text_cur;
        const unsigned long long base = run ? atomicAdd(cur, run) : 0ull;
        for (uint32_t w = 0; w < nw; ++w) r[w] += base;
    }
    __syncthreads();
    const Res out{B.rs[0][wid] + a - fa, B.rs[1][wid] + b - nlm, B.rs[2][wid] + c - lmb};
    __syncthreads();   // the offsets are read before the next reservation overwrites them
    return out;
}

// The L bases of a reserved FASTA record ">0\n...\n" at offset o, or nullptr past the arena.
__device__ __forceinline__ char* fasta_at(const Sink& sk, unsigned long long o, uint32_t L) {
    if (o + L + 4 > sk.fasta_cap) { atomicOr(sk.oflow, DERR_OUT_OVERFLOW); return nullptr; }
    char* p = sk.fasta + o;
    p[0] = '>'; p[1] = '0'; p[2] = '\n'; p[3 + L] = '\n';
    return p + 3;
}

__device__ __forceinline__ uint32_t lane_lt() { uint32_t m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

// Appends val(ls) for every local slot ls < per with pred(ls) to the shared work list wl
// (order unspecified; compact appends ls itself).  All threads of the CTA must call it;
// blockDim is a multiple of 32.
template <typename Pred, typename Val>
__device__ __forceinline__ void compact_to(uint32_t per, uint32_t* wl, uint32_t* n, Pred pred, Val val) {
    const uint32_t nt = blockDim.x;
    for (uint32_t base = 0; base < per; base += nt) {
        const uint32_t ls = base + threadIdx.x;
        const bool p = ls < per && pred(ls);
        const uint32_t m = __ballot_sync(0xffffffffu, p);
        uint32_t at = 0;
        if ((threadIdx.x & 31) == 0 && m) at = atomicAdd(n, (uint32_t)__popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (p) wl[at + __popc(m & lane_lt())] = val(ls);
    }
}
template <typename Pred>
__device__ __forceinline__ void compact(uint32_t per, uint32_t* wl, uint32_t* n, Pred pred) {
    compact_to(per, wl, n, pred, [](uint32_t ls) { return ls; });
}

template <int MODE> __device__ __forceinline__ void tsync() {
    if constexpr (MODE == CLUSTER) cg::this_cluster().sync();
    else __syncthreads();
}

template <int W>
__device__ __forceinline__ Kmer<W> phi_kmer(const KOps<W>& ops) {   // all-T k-mer, include/Discontinuity_Graph.hpp:44-49
    Kmer<W> x;
    if constexpr (W == 1) x.lo = ops.mask;
    else if constexpr (W == 2) { x.lo = ~0ull; x.hi = ops.mhi; }
    else {
#pragma unroll
        for (int j = 0; j < W - 1; ++j) x.w[j] = ~0ull;
        x.w[W - 1] = ops.mhi;
    }
    return x;
}

template <int W>
__device__ __forceinline__ void put_key(uint64_t out[4], const Kmer<W>& x) {
#pragma unroll
    for (int j = 0; j < 4; ++j) out[j] = j < W ? x.word(j < W ? j : 0) : 0ull;
}

// A vertex in walk direction: its directed k-mer, the reverse complement, and its slot.
template <int W> struct DV { Kmer<W> d, r; uint32_t slot; uint64_t st; };   // st: the slot's state word

// Oriented vertex leaving slot s through `side`: the directed form is the canonical
// k-mer when leaving through the back side (Directed_Vertex exit_side, :295-299).
template <int W, int MODE>
__device__ __forceinline__ DV<W> dv_at(const Tab<W, MODE>& T, const KOps<W>& ops, uint32_t s, int side) {
    const Kmer<W> x = T.key(s), xr = ops.rc(x);
    const uint64_t st = T.ld_st(s);
    return side == BACK ? DV<W>{x, xr, s, st} : DV<W>{xr, x, s, st};
}

// One walk step out of v through `side` (which must hold a single passing edge):
// the next vertex (with its state word) and the side it is entered by.
template <int W, int MODE>
__device__ __forceinline__ bool step_inline(const Tab<W, MODE>& T, const KOps<W>& ops, uint32_t fth, DV<W>& v, int side, int& s_in) {
    const uint32_t e = ef_edge_at(st_ef(v.st), side, fth);
    const uint32_t b = side == BACK ? e : 3 - e;
    ops.push_back(v.d, b);
    ops.push_front(v.r, 3 - b);
    const bool c = v.d < v.r;
    uint64_t stv = 0;
    const uint32_t u = T.find(c ? v.d : v.r, stv);
    if (u == NONE) return false;
    v.slot = u;
    v.st = stv;
    s_in = c ? FRONT : BACK;
    return true;
}

template <int W, int MODE>
__device__ __forceinline__ bool step(const Tab<W, MODE>& T, const KOps<W>& ops, uint32_t fth, DV<W>& v, int side, int& s_in) {
    return step_inline(T, ops, fth, v, side, s_in);
}

// A homopolymer b^k (b in {A, C}; x canonical) whose back side holds only its self-loop
// and whose front side holds at most one edge: seeded on its own, the reference's walk
// records it as a one-vertex cycle.
template <int W>
__device__ __forceinline__ bool looped_homopolymer(const KOps<W>& ops, const Kmer<W>& x, uint32_t ef, uint32_t fth) {
    const uint32_t eb = ef_edge_at(ef, BACK, fth);
    return eb < 2 && ef_count(ef, FRONT, fth) <= 1 && ops.is_homopolymer(x, eb);
}

// Bytes written one at a time in address order (rising or falling), gathered into
// whole 8-byte words: one store per aligned word the run covers, byte stores only
// at its two ragged ends.
struct WordWriter {
    unsigned long long base = ~0ull;   // address of the aligned word being gathered
    unsigned long long w = 0;
    uint32_t mask = 0;                 // bytes of that word gathered so far
    __device__ __forceinline__ void flush() {
        if (!mask) return;
        if (mask == 0xFFu) *(unsigned long long*)base = w;
        else
            for (uint32_t b = 0; b < 8; ++b)
                if ((mask >> b) & 1) ((char*)base)[b] = (char)(w >> (8 * b));
        mask = 0; w = 0;
    }
    __device__ __forceinline__ void put(char* a, char c) {
        const unsigned long long ad = (unsigned long long)a, wb = ad & ~7ull;
        if (wb != base) { flush(); base = wb; }
        const uint32_t o = (uint32_t)(ad & 7);
        w |= (unsigned long long)(uint8_t)c << (8 * o);
        mask |= 1u << o;
    }
};

// Writes the label of the path of n vertices that starts at v (in walk direction).  With
// links (one-CTA tables of at most LINK_SLOTS slots) every step follows the link W1 stored
// for the side it leaves by -- every side inside a path or an isolated cycle has one -- and
// appends the base of the side's single edge, with no table lookup.
template <int W, int MODE>
__device__ void write_path(const Tab<W, MODE>& T, const KOps<W>& ops, uint32_t fth, DV<W> v, int side, uint32_t n,
                           char* dst, bool rev, bool mark, bool links = false) {
    const uint32_t k = ops.k, L = n + k - 1;
    WordWriter ww;
    auto put = [&](uint32_t i, uint32_t b) {
        if (!rev) ww.put(dst + i, "ACGT"[b]);
        else ww.put(dst + (L - 1 - i), "ACGT"[3 - b]);
    };
    if (dst) for (uint32_t i = 0; i < k; ++i) put(i, ops.base(v.d, i));
    if (mark) T.or_meta(v.slot, M_VISITED);
    for (uint32_t t = 1; t < n; ++t) {
        int s_in;
        uint32_t b;
        if (links) {
            const uint32_t f = side_field(T.ld_meta(v.slot), side);
            if (!(f & 1)) break;
            const uint32_t e = ef_edge_at(st_ef(v.st), side, fth);
            b = side == BACK ? e : 3 - e;
            v.slot = (f >> 1) & (LINK_SLOTS - 1);
            s_in = (int)(f >> 13);
            v.st = T.ld_st(v.slot);
        } else {
            if (!step(T, ops, fth, v, side, s_in)) break;
            b = ops.last_base(v.d);
        }
        if (dst) put(k - 1 + t, b);
        if (mark) T.or_meta(v.slot, M_VISITED);
        side = 1 - s_in;
    }
    if (dst) ww.flush();
}

// A one-k-mer cycle (a self-looped homopolymer seeded on its own) at reserved FASTA offset o.
template <int W, int MODE>
__device__ void write_kmer_cycle(const Tab<W, MODE>& T, const KOps<W>& ops, uint32_t s, Block& B, unsigned long long o) {
    char* p = fasta_at(B.sk, o, ops.k);
    if (p) { const Kmer<W> x = T.key(s); for (uint32_t i = 0; i < ops.k; ++i) p[i] = "ACGT"[ops.base(x, i)]; }
    atomicAdd(&B.trivial, 1ull); atomicAdd(&B.icc, 1ull);
}

template <int W>
__device__ __forceinline__ bool local_empty(const unsigned long long* lkeys, uint32_t ls) {
    // the key's highest word (16 bytes per slot's key part for k <= 63, 32 beyond)
    return lkeys[(size_t)ls * (W <= 2 ? 2 : 4) + (W - 1)] == EMPTY;
}
// index of local slot ls's state word in the state array (interleaved with the keys for k <= 31)
template <int W> __device__ __forceinline__ uint32_t sti(uint32_t ls) { return W == 1 ? 2 * ls : ls; }

struct EndInfo { uint32_t slot; uint32_t term; bool canon; };   // a path end in walk direction

// The bases of one weak super k-mer, MSB-first from its first base (base 0 at bits
// 63:62 of w[0]): 2 words for k <= 31 (a record holds at most 2(k-1)-l+2 <= 61
// bases), 4 for k <= 63 (<= 125), 6 for k <= 95 (<= 189), 8 for k <= 127 (<= 253).
// The packed stream carries 4 words of padding, which covers the unconditional loads
// of k <= 63; wider records load only the words that hold their len bases.
template <int W>
struct RecWords {
    static constexpr int NW = 2 * W;
    uint64_t w[NW];
    __device__ __forceinline__ RecWords() {}
    __device__ __forceinline__ RecWords(const uint64_t* __restrict__ s, uint32_t pos, bool has, uint32_t len = 0) {
        const uint64_t q = pos >> 5;
        const uint32_t sh = 2 * (pos & 31);
        const uint32_t last = ((pos & 31) + (len ? len : 1) - 1) >> 5;   // the record's last word, from q
        uint64_t a[NW + 1];
#pragma unroll
        for (int i = 0; i <= NW; ++i) a[i] = has && (W <= 2 || (uint32_t)i <= last) ? __ldg(s + q + i) : 0ull;
#pragma unroll
        for (int i = 0; i < NW; ++i) w[i] = sh ? (a[i] << sh) | (a[i + 1] >> (64 - sh)) : a[i];
    }
    // the words of the record held by lane j of the warp
    __device__ __forceinline__ RecWords from_lane(uint32_t j) const {
        RecWords r;
#pragma unroll
        for (int i = 0; i < NW; ++i) r.w[i] = __shfl_sync(0xffffffffu, w[i], j);
        return r;
    }
    __device__ __forceinline__ uint64_t word(uint32_t i) const {   // word i, 0 past the end
        uint64_t v = 0;
#pragma unroll
        for (int x = 0; x < NW; ++x) v = i == (uint32_t)x ? w[x] : v;
        return v;
    }
    __device__ __forceinline__ uint64_t bases64(uint32_t i) const {   // bases i .. i+31, base i at 63:62
        const uint32_t j = i >> 5, o = 2 * (i & 31);
        const uint64_t a = word(j);
        return o ? (a << o) | (word(j + 1) >> (64 - o)) : a;
    }
    __device__ __forceinline__ uint32_t base(uint32_t i) const { return (uint32_t)(word(i >> 5) >> (62 - 2 * (i & 31))) & 3; }
    // the k-mer at offset idx of a record of len bases, its predecessor and successor base
    // (BASE_E at the record's ends)
    __device__ __forceinline__ void kmer_at(uint32_t k, uint32_t idx, uint32_t len, Kmer<W>& x, uint32_t& pred,
                                            uint32_t& succ) const {
        if constexpr (W == 1) {
            const uint64_t win = bases64(idx);   // idx + k <= 61 < 64: the k-mer and its successor
            x.lo = win >> (64 - 2 * k);
            succ = idx + k == len ? BASE_E : (uint32_t)(win >> (62 - 2 * k)) & 3;
        } else if constexpr (W == 2) {
            const uint32_t nh = k - 32;          // bases in the high word
            x.hi = bases64(idx) >> (64 - 2 * nh);
            x.lo = bases64(idx + nh);
            succ = idx + k == len ? BASE_E : base(idx + k);
        } else {
            const uint32_t nh = k - 32 * (W - 1);   // bases in the highest word
            x.w[W - 1] = bases64(idx) >> (64 - 2 * nh);
#pragma unroll
            for (int j = W - 2; j >= 0; --j) x.w[j] = bases64(idx + nh + 32 * (W - 2 - j));
            succ = idx + k == len ? BASE_E : base(idx + k);
        }
        pred = idx == 0 ? BASE_E : base(idx - 1);
    }
};

// A path of n vertices from v0 (leaving through side0) to vlast, written into space
// reserved by reserve_warp: a trivial maximal unitig at FASTA offset fo, or an lm-tig
// (lm: one end exits the subgraph) as record idx with its label at offset off.
// The label of a path whose bases the walk kept: the walk's first k-mer, then one base
// per step; `skip` leading bases are not part of the path (a one-k-mer cycle at its start).

// The walk's bases as a little-endian 2-bit array over four words: base j at bits
// 2 (j & 31) of word j >> 5 (first k-mer, then up to 64 steps: at most 127 bases).
struct WalkSeq { uint64_t w0, w1, w2, w3; };
__device__ __forceinline__ uint64_t rev_bases(uint64_t x) {   // reverses the order of 32 2-bit bases
    const uint64_t r = __brevll(x);
    return ((r >> 1) & 0x5555555555555555ull) | ((r & 0x5555555555555555ull) << 1);
}
template <int W>
__device__ __forceinline__ WalkSeq walk_seq(uint32_t k, const Kmer<W>& first, uint64_t s0, uint64_t s1) {
    WalkSeq q;
    if constexpr (W == 1) {   // k <= 31
        const uint32_t sh = 2 * k;
        const uint64_t f = rev_bases(first.lo) >> (64 - sh);
        q.w0 = f | (s0 << sh); q.w1 = (s0 >> (64 - sh)) | (s1 << sh); q.w2 = s1 >> (64 - sh); q.w3 = 0;
    } else if constexpr (W == 2) {   // 33 <= k <= 63: hi holds the first k - 32 bases
        const uint32_t sh = 2 * (k - 32);
        const uint64_t h = rev_bases(first.hi) >> (64 - sh), lo = rev_bases(first.lo);
        q.w0 = h | (lo << sh); q.w1 = (lo >> (64 - sh)) | (s0 << sh);
        q.w2 = (s0 >> (64 - sh)) | (s1 << sh); q.w3 = s1 >> (64 - sh);
    } else {                  // k > 63 keeps no buffered labels (first k-mer + steps exceed 128 bases)
        q.w0 = q.w1 = q.w2 = q.w3 = 0;
    }
    return q;
}
// bases j .. j+7 (j + 8 <= 128), base j in bits 1:0
__device__ __forceinline__ uint32_t seq_get16(const WalkSeq& q, uint32_t j) {
    const uint32_t w = j >> 5, o = 2 * (j & 31);
    const uint64_t a = w == 0 ? q.w0 : w == 1 ? q.w1 : w == 2 ? q.w2 : q.w3;
    const uint64_t b = w == 0 ? q.w1 : w == 1 ? q.w2 : w == 2 ? q.w3 : 0ull;
    const uint64_t v = o ? ((a >> o) | (b << (64 - o))) : a;
    return (uint32_t)v & 0xFFFFu;
}
// character tables for __byte_perm: byte b is the character of base b (or of its complement)
constexpr uint32_t CH_FWD = 0x54474341u;   // A C G T
constexpr uint32_t CH_CMP = 0x41434754u;   // T G C A
__device__ __forceinline__ uint32_t sel4(uint32_t x) {   // four 2-bit bases -> one selector nibble each
    return (x & 3u) | ((x & 0xCu) << 2) | ((x & 0x30u) << 4) | ((x & 0xC0u) << 6);
}
__device__ __forceinline__ uint64_t chars8(uint32_t x16, uint32_t table) {
    return (uint64_t)__byte_perm(table, 0, sel4(x16 & 0xFFu)) | ((uint64_t)__byte_perm(table, 0, sel4(x16 >> 8)) << 32);
}
__device__ __forceinline__ uint32_t rev8bases(uint32_t x16) {   // reverses the order of 8 2-bit bases
    const uint32_t r = __brev(x16) >> 16;
    return ((r >> 1) & 0x5555u) | ((r & 0x5555u) << 1);
}

// Output byte i is base skip + i (forward), or the complement of base skip + L - 1 - i
// (rev); written in address order, eight characters per aligned 8-byte store.
template <int W>
__device__ void write_buffered(const KOps<W>& ops, const Kmer<W>& first, unsigned long long steps0,
                               unsigned long long steps1, uint32_t skip, uint32_t L, char* dst, bool rev) {
    if (!dst || W > 2) return;
    const WalkSeq q = walk_seq<W>(ops.k, first, steps0, steps1);
    const uint32_t table = rev ? CH_CMP : CH_FWD;
    auto one = [&](uint32_t i) {
        const uint32_t b = seq_get16(q, rev ? skip + L - 1 - i : skip + i) & 3u;
        dst[i] = (char)(table >> (8 * b));
    };
    const uint32_t off = (uint32_t)((unsigned long long)dst & 7);
    const uint32_t head = off ? (L < 8 - off ? L : 8 - off) : 0;
    uint32_t i = 0;
    for (; i < head; ++i) one(i);
    for (; i + 8 <= L; i += 8) {
        const uint32_t x = rev ? rev8bases(seq_get16(q, skip + L - 8 - i)) : seq_get16(q, skip + i);
        *(unsigned long long*)(dst + i) = chars8(x, table);
    }
    for (; i < L; ++i) one(i);
}

template <int W, int MODE>
__device__ void write_emitted_path(const SubgraphArgs& a, const Tab<W, MODE>& T, const KOps<W>& ops, const DV<W>& v0,
                                   int side0, uint32_t n, const DV<W>& vlast, EndInfo st, EndInfo en, bool seed_canon,
                                   Block& B, bool lm, unsigned long long fo, unsigned long long idx,
                                   unsigned long long off, bool buffered, unsigned long long steps0,
                                   unsigned long long steps1, const Kmer<W>& first, uint32_t skip, bool links) {
    const uint32_t k = ops.k, fth = a.fth;
    const uint32_t L = n + k - 1;
    if (!lm) {
        // trivial maximal unitig in canonical orientation (Maximal_Unitig_Scratch::finalize, :200-222)
        const bool rev = vlast.r < v0.d;   // rc(last k-mer) < first k-mer
        char* p = fasta_at(B.sk, fo, L);
        if (buffered) write_buffered(ops, first, steps0, steps1, skip, L, p, rev);
        else write_path(T, ops, fth, v0, side0, n, p, rev, true, links);
        atomicAdd(&B.trivial, 1ull);
        return;
    }
    // lm-tig oriented by its first-inserted vertex (finalize_weak, :225-233; Unitig_File add, include/Unitig_File.hpp:338-359)
    const bool rev = !seed_canon;
    const EndInfo eu = rev ? en : st, ev = rev ? st : en;
    const bool u_first_canon = rev ? !en.canon : st.canon;     // label's first k-mer canonical?
    const bool v_last_canon = rev ? !st.canon : en.canon;      // label's last k-mer canonical?
    const Sink& sk = B.sk;
    atomicAdd(&B.lmtig, 1ull);
    const bool fits = idx < sk.lm_cap && off + L <= sk.lm_text_cap;
    if (!fits) atomicOr(sk.oflow, DERR_OUT_OVERFLOW);
    if (buffered) write_buffered(ops, first, steps0, steps1, skip, L, fits ? sk.lm_text + off : nullptr, rev);
    else write_path(T, ops, fth, v0, side0, n, fits ? sk.lm_text + off : nullptr, rev, true, links);
    if (!fits) return;
    LmtigOut o;
    const Kmer<W> phi = phi_kmer(ops);
    const bool u_exit = eu.term == T_EXIT, v_exit = ev.term == T_EXIT;
    put_key(o.u, u_exit ? T.key(eu.slot) : phi);
    put_key(o.v, v_exit ? T.key(ev.slot) : phi);
    const uint32_t s_u_back = u_exit ? (u_first_canon ? 1u : 0u) : 1u;
    const uint32_t s_v_back = v_exit ? (v_last_canon ? 0u : 1u) : 1u;
    o.label_off = off; o.label_len = L; o.g = (uint16_t)sk.g;
    o.flags = (uint8_t)(s_u_back | (s_v_back << 1) | ((!u_exit) << 2) | ((!v_exit) << 3));
    o.pad = 0;
    sk.lm[idx] = o;
}

// rank/nranks: this CTA's position in its cluster; per: slots owned by one CTA.
// Merges the identical records of [q0, q1) (one-CTA tables, k <= 31, records of at most
// 60 bases).  A table of per / 2 entries of 32 bytes is laid over the still unused vertex
// table (lkeys): key = the record's bases, MSB-first, in two words with its length and
// discontinuity marks in the low byte of the second (all ones in both: empty -- a real
// second word never ends in 0xFF, since lengths stay below 63); value = the smallest
// (stream position << 32 | index from q0) of its copies and their count.  Every probe is
// a 16-byte compare-and-swap, which returns the entry's whole key in one atomic step, so
// no reader sees half a key.  On success wl holds one entry per distinct record -- the
// index from q0 of its first copy in the stream | min(count, 15) << 20 -- and B.wl_n their
// number; false (nothing merged) when the table filled up.  All threads of the CTA call it.
__device__ bool dedup_records(const SubgraphArgs& a, Block& B, uint32_t q0, uint32_t q1, uint32_t per,
                              unsigned long long* lkeys, uint32_t* wl) {
    typedef Mem<LOCAL> M;
    const uint32_t tid = threadIdx.x, nt = blockDim.x, D = per / 2;
    for (uint32_t e = tid; e < D; e += nt) {
        lkeys[4 * e] = EMPTY; lkeys[4 * e + 1] = EMPTY; lkeys[4 * e + 2] = ~0ull; lkeys[4 * e + 3] = 0;
    }
    if (tid == 0) { B.dd_over = 0; B.wl_n = 0; }
    __syncthreads();
    const uint32_t base = smem_addr(lkeys);
    const uint32_t bound = D > 256 ? D / 4 : D;
    for (uint32_t r = q0 + tid; r < q1; r += nt) {
        if (*(volatile uint32_t*)&B.dd_over) break;
        const uint64_t rec = a.recs[r];
        const uint32_t len = rec_len(rec), pos = rec_pos(rec);
        const RecWords<1> rw(a.packed, pos, true);
        const uint64_t k0 = len >= 32 ? rw.w[0] : rw.w[0] & ~(~0ull >> (2 * len));
        const uint64_t k1 = (len > 32 ? rw.w[1] & ~(~0ull >> (2 * (len - 32))) : 0ull) | (uint64_t)len |
                            ((uint64_t)rec_ld(rec) << 6) | ((uint64_t)rec_rd(rec) << 7);
        const uint64_t z = (k0 ^ (k1 * 0xC2B2AE3D27D4EB4Full)) * 0x9E3779B97F4A7C15ull;
        uint32_t h = (uint32_t)(((z >> 32) * D) >> 32);
        bool done = false;
        for (uint32_t p = 0; p < bound; ++p) {
            const uint32_t ea = base + h * 32;
            uint64_t o0, o1;
            M::cas128(ea, EMPTY, EMPTY, k0, k1, o0, o1);
            if ((o0 == EMPTY && o1 == EMPTY) || (o0 == k0 && o1 == k1)) {
                const uint64_t pi = ((uint64_t)pos << 32) | (r - q0);
                asm volatile("red.shared.min.u64 [%0], %1;" :: "r"(ea + 16), "l"(pi) : "memory");
                asm volatile("red.shared.add.u32 [%0], %1;" :: "r"(ea + 24), "r"(1u) : "memory");
                done = true;
                break;
            }
            if (++h == D) h = 0;
        }
        if (!done) { atomicOr(&B.dd_over, 1u); break; }
    }
    __syncthreads();
    if (*(volatile uint32_t*)&B.dd_over) return false;   // its own flag: the caller resets B.overflow next
    compact_to(D, wl, &B.wl_n, [&](uint32_t e) { return lkeys[4 * e + 1] != EMPTY; }, [&](uint32_t e) {
        const uint32_t c = (uint32_t)lkeys[4 * e + 3];
        return ((uint32_t)lkeys[4 * e + 2] & 0xFFFFFu) | ((c < 15u ? c : 15u) << 20);
    });
    __syncthreads();
    return true;
}

template <int W, int MODE>
__device__ void run_subgraph(const SubgraphArgs& a, const Tab<W, MODE>& T, Block& B, Block* Bc,
                             uint32_t g, uint32_t rank, uint32_t nranks, uint32_t per,
                             unsigned long long* lkeys, unsigned long long* lst, uint32_t* lmeta, uint32_t* wl) {
    long long clk[6];
    clk[0] = clock64();
    const KOps<W> ops(a.k);
    const uint32_t k = a.k, fth = a.fth;
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    const uint32_t base_slot = rank * per;
    const uint32_t r0 = a.bucket_off[g], r1 = a.bucket_off[g + 1];
    // this CTA's share of the subgraph's records (all of them for one-CTA tables)
    const uint32_t q0 = r0 + (uint32_t)((uint64_t)(r1 - r0) * rank / nranks);
    const uint32_t q1 = r0 + (uint32_t)((uint64_t)(r1 - r0) * (rank + 1) / nranks);
    // the build's items: the records [q0, q1), or the distinct ones in wl when merged
    uint32_t n_items = q1 - q0;
    bool from_list = false;
    if constexpr (W == 1 && MODE == LOCAL) {
        if (a.dedup && n_items >= 64 && n_items < (1u << 20) && dedup_records(a, B, q0, q1, per, lkeys, wl)) {
            from_list = true;
            n_items = B.wl_n;   // only the merge writes this count
        }
    }
    // One-table modes keep two lists in wl, one growing from each end: the build appends
    // the slots it claims at the top (the merged records, if any, hold the bottom), and
    // W1, reading that list, appends the path ends at the bottom -- no pass over every
    // slot to compact them.  A list that would run into the other falls back to a
    // compaction pass.  Cluster tables compact per CTA as before.
    constexpr bool LISTS = MODE != CLUSTER;
    const uint32_t cap_fresh = per - (from_list ? n_items : 0u);

    for (uint32_t s = tid; s < per; s += nt) {
        if constexpr (W == 1) lkeys[2 * s] = EMPTY;
        else if constexpr (W == 2) { lkeys[2 * s] = EMPTY; lkeys[2 * s + 1] = EMPTY; }
        else { lkeys[4 * s] = EMPTY; lkeys[4 * s + 1] = EMPTY; lkeys[4 * s + 2] = EMPTY; lkeys[4 * s + 3] = EMPTY; }
        lst[sti<W>(s)] = ST_INIT;
        lmeta[s] = 0;
    }
    if (tid == 0) {
        B.inserted = 0; B.overflow = 0; B.covered = 0;
        B.fresh_n = 0; B.w1_n = 0; B.end_n = 0; B.cyc_n = 0;
        B.vertices = B.isolated = B.phantom = B.trivial = B.icc = B.lmtig = 0;
        sink_for(a, g, B.sk);
    }
    tsync<MODE>();

    // ---------------- build ----------------
    const uint32_t limit = (uint32_t)(((uint64_t)per * a.load_limit_pct) / 100);
    uint32_t n_fresh = 0;   // vertices this thread inserted
    // HT_Router::update of one k-mer instance at stream position p (idx-th of its record):
    // edges from its predecessor / successor bases, the self-loop rule against the
    // previous k-mer's canonical form, and the record's entrance / exit marks.
    auto insert = [&](const Kmer<W>& fw, const Kmer<W>& rc, const Kmer<W>& pred_can, uint32_t idx, uint32_t pred,
                      uint32_t succ, uint32_t p, bool l_mark, bool r_mark, uint32_t m, uint32_t& slot_out,
                      bool& fresh_out) -> bool {
        const bool canon = fw < rc;
        const Kmer<W> can = canon ? fw : rc;
        uint32_t front = canon ? pred : compb(succ);
        uint32_t back = canon ? succ : compb(pred);
        if (idx > 0 && can == pred_can) { if (canon) front = BASE_E; else back = BASE_E; }
        uint32_t owner, h;
        T.place(can, owner, h);
        bool fresh;
        uint32_t s;
        if constexpr (W == 1) {
            s = T.upsert(can, owner, h, front, back, p, m, fresh);
        } else {
            uint64_t seen = ST_INIT;
            s = T.find_or_insert(can, owner, h, fresh, seen);
            if (s != NONE) T.update_state(s, front, back, p, m, seen);
        }
        if (s == NONE) { atomicOr(&B.overflow, 1u); return false; }
        n_fresh += fresh;
        slot_out = s; fresh_out = fresh;
        uint32_t disc = 0;
        if (l_mark) disc |= canon ? M_DISC_F : M_DISC_B;      // entrance side
        if (r_mark) disc |= canon ? M_DISC_B : M_DISC_F;      // exit side
        if (disc) T.mark_disc(s, disc);
        return true;
    };
    // Each warp takes 32 items (records, or distinct records with their multiplicity) at
    // a time; lane i loads item i's record and its bases once (<= 2 words for k <= 31, <= 4
    // for k <= 63).  The records' k-mer instances are then dealt out in runs of up to RUN
    // consecutive instances of one record, 32 runs per round, so every lane has work
    // whatever the record lengths: the lane of run t finds its record from the bit mask of
    // the records starting in the round and takes that record's words (and multiplicity)
    // from its owner lane by shuffles.  A run's first k-mer is cut from the record's words;
    // each next one rolls in one base (its reverse complement, predecessor base and the
    // previous canonical k-mer come from the instance before).  k <= 31 deals single
    // instances: its records are short (<= 61 bases), and runs left lanes idle there.
    {
        constexpr uint32_t RUN = W == 1 ? 1 : 4;
        const uint32_t lane = tid & 31, nwarps = nt >> 5;
        const uint32_t le_mask = lane_lt() | (1u << lane);
        bool stop = false;
        for (uint32_t rb = (tid >> 5) * 32; rb < n_items && !stop; rb += nwarps * 32) {
            const uint32_t i = rb + lane;
            const bool has = i < n_items;
            const uint32_t item = has && from_list ? wl[i] : i;
            const uint64_t rec = has ? a.recs[q0 + (from_list ? item & 0xFFFFFu : item)] : 0ull;
            const uint32_t mult = from_list ? item >> 20 : 1u;
            const uint32_t ninst = has ? rec_len(rec) - k + 1 : 0u;
            const uint32_t nrun = (ninst + RUN - 1) / RUN;
            uint32_t incl = nrun;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, incl, d);
                if (lane >= (uint32_t)d) incl += y;
            }
            const uint32_t P = incl - nrun;                       // first run of record `lane`
            const uint32_t total = __shfl_sync(FULL, incl, 31);
            const RecWords<W> rw(a.packed, has ? rec_pos(rec) : 0u, has, has ? rec_len(rec) : 0u);
            uint32_t started = 0;                                 // records started before the round
            for (uint32_t t0 = 0; t0 < total; t0 += 32) {
                const uint32_t bit = (has && P >= t0 && P < t0 + 32) ? 1u << (P - t0) : 0u;
                const uint32_t smask = __reduce_or_sync(FULL, bit);
                const uint32_t jj = started + __popc(smask & le_mask);
                const uint32_t j = jj ? min(jj - 1, 31u) : 0u;   // the record of run t0 + lane
                started += __popc(smask);
                const uint64_t rj = __shfl_sync(FULL, rec, j);
                const uint32_t Pj = __shfl_sync(FULL, P, j);
                const uint32_t mj = __shfl_sync(FULL, mult, j);
                const RecWords<W> xw = rw.from_lane(j);
                const uint32_t t = t0 + lane;
                const uint32_t len = rec_len(rj);
                const uint32_t idx0 = t < total ? (t - Pj) * RUN : 0u;
                const uint32_t cnt = t < total ? min(RUN, len - k + 1 - idx0) : 0u;
                bool ok = true;
                Kmer<W> fw{}, rc{}, pc{};
                uint32_t pred = 0, succ = 0;
                if (cnt) {
                    xw.kmer_at(k, idx0, len, fw, pred, succ);
                    rc = ops.rc(fw);
                    pc = fw;
                    if (idx0 > 0) {   // the previous k-mer and its reverse complement, from fw and rc
                        Kmer<W> pf = fw, pr = rc;
                        ops.push_front(pf, pred);
                        ops.push_back(pr, 3 - pred);
                        pc = pf < pr ? pf : pr;
                    }
                }
#pragma unroll 1
                for (uint32_t r = 0; r < RUN; ++r) {   // uniform over the warp
                    bool fr = false;
                    uint32_t fs = 0;
                    if (r < cnt && ok) {
                        const uint32_t idx = idx0 + r;
                        if (r > 0) {   // roll in the base after the previous k-mer
                            pc = fw < rc ? fw : rc;
                            pred = ops.first_base(fw);
                            ops.push_back(fw, succ);
                            ops.push_front(rc, 3 - succ);
                            succ = idx + k == len ? BASE_E : xw.base(idx + k);
                        }
                        ok = insert(fw, rc, pc, idx, pred, succ, rec_pos(rj) + idx, idx == 0 && rec_ld(rj),
                                    idx + k == len && rec_rd(rj), mj, fs, fr);
                    }
                    if constexpr (LISTS) {   // the claimed slots, at the top of wl (one atomic per warp and step)
                        const uint32_t fm = __ballot_sync(FULL, fr);
                        if (fm) {
                            uint32_t b0 = 0;
                            if (lane == 0) b0 = atomicAdd(&B.fresh_n, (uint32_t)__popc(fm));
                            b0 = __shfl_sync(FULL, b0, 0);
                            const uint32_t jx = b0 + __popc(fm & lane_lt());
                            if (fr && jx < cap_fresh) wl[per - 1 - jx] = fs;
                        }
                    }
                }
                // a failed insert (table full) stops the build: warp-uniform, between rounds
                if (__any_sync(FULL, !ok || *(volatile uint32_t*)&B.overflow)) { stop = true; break; }
            }
        }
    }
    // fresh vertices are counted per inserting CTA (records, hence inserts, are spread
    // evenly, so one CTA's count stands for one sub-table's load) and summed once: a table
    // past its load limit is retried larger (one that fills up stops the build earlier,
    // through an insert that exhausts its probe bound)
    for (int d = 16; d; d >>= 1) n_fresh += __shfl_down_sync(0xffffffffu, n_fresh, d);
    if ((tid & 31) == 0 && n_fresh) atomicAdd(&B.inserted, n_fresh);
    __syncthreads();
    bool overflow;
    if constexpr (MODE == CLUSTER) {
        if (tid == 0 && B.inserted > limit) B.overflow = 1;
        // one CTA's overflow is the whole cluster's
        __syncthreads();
        if (tid == 0 && B.overflow && Bc != &B) atomicOr(&Bc->overflow, 1u);
        tsync<MODE>();
        overflow = *(volatile uint32_t*)&Bc->overflow;
    } else {   // one table: every thread reads the build's final counts
        overflow = *(volatile uint32_t*)&B.overflow || *(volatile uint32_t*)&B.inserted > limit;
    }
    if (overflow) {
        if (rank == 0 && tid == 0) {
            const unsigned long long i = atomicAdd(&a.cnt->retry_count, 1ull);
            a.retry[i] = g;
        }
        tsync<MODE>();   // no CTA leaves while another may still read its shared memory
        return;
    }

    clk[1] = clock64();
    // ---------------- W1: termination of every side ----------------
    // its list: the slots the build claimed (top of wl), else a compaction (bottom)
    const uint32_t n_claimed = LISTS ? *(volatile uint32_t*)&B.fresh_n : 0u;
    const bool l1_top = LISTS && n_claimed <= cap_fresh;
    if (!l1_top) {
        compact(per, wl, &B.w1_n, [&](uint32_t ls) { return !local_empty<W>(lkeys, ls); });
        __syncthreads();
    }
    const uint32_t n1 = l1_top ? n_claimed : *(volatile uint32_t*)&B.w1_n;
    const uint32_t cap_end = per - n1;   // path ends go to the other end of wl
    const bool links = MODE == LOCAL && per <= LINK_SLOTS;
    uint32_t n_vert = 0, n_iso = 0, n_phantom = 0;   // this thread's vertices (summed once per warp)
    for (uint32_t base = 0; base < n1; base += nt) {   // uniform over the CTA: warps append path ends together
      const uint32_t i = base + tid;
      bool is_end = false;
      uint32_t ls = 0;
      if (i < n1) do {
        ls = wl[l1_top ? per - 1 - i : i];
        const uint32_t s = base_slot + ls;
        const uint32_t ef = st_ef(lst[sti<W>(ls)]);
        uint32_t meta = lmeta[ls];
        const uint32_t cf = ef_count(ef, FRONT, fth), cb = ef_count(ef, BACK, fth);
        ++n_vert;
        if (cf == 0 && cb == 0) {
            ++n_iso;
            if (meta & (M_DISC_F | M_DISC_B)) ++n_phantom;
            lmeta[ls] = meta | M_ISO;
            break;
        }
        const Kmer<W> x = T.key(s);
        const Kmer<W> xr = ops.rc(x);
        for (int side = 0; side < 2; ++side) {
            const uint32_t e = ef_edge_at(ef, side, fth);
            uint32_t term = T_OK, link = 0;
            if (e == BASE_N) term = T_BRANCHED;
            else if (e == BASE_E) term = (meta & (side == FRONT ? M_DISC_F : M_DISC_B)) ? T_EXIT : T_DEAD;
            else {
                Kmer<W> y, yr;
                if (side == BACK) { y = x; ops.push_back(y, e); yr = xr; ops.push_front(yr, 3 - e); }
                else { y = xr; ops.push_back(y, 3 - e); yr = x; ops.push_front(yr, e); }
                const bool yc = y < yr;
                uint64_t ust = 0;
                const uint32_t u = T.find(yc ? y : yr, ust);
                const int s_in = yc ? FRONT : BACK;
                if (u == NONE) { atomicOr(a.err, DERR_MISSING_KEY); term = T_CROSSED; }
                else if (u == s) term = T_CROSSED;                                        // self-loop
                else if (ef_count(st_ef(ust), s_in, fth) > 1) term = T_CROSSED;    // branching entrance
                else if (links) link = 1u | (u << 1) | ((uint32_t)s_in << 13);
            }
            meta |= side_bits(link ? link : term << 1, side);
        }
        lmeta[ls] = meta;
        is_end = term_of(meta, FRONT) != T_OK || term_of(meta, BACK) != T_OK;
      } while (false);
      if constexpr (LISTS) {
        const uint32_t em = __ballot_sync(FULL, is_end);
        if (em) {
            uint32_t b0 = 0;
            if ((tid & 31) == 0) b0 = atomicAdd(&B.end_n, (uint32_t)__popc(em));
            b0 = __shfl_sync(FULL, b0, 0);
            const uint32_t jx = b0 + __popc(em & lane_lt());
            if (is_end && jx < cap_end) wl[l1_top ? jx : per - 1 - jx] = ls;
        }
      }
    }
    for (int d = 16; d; d >>= 1) {
        n_vert += __shfl_down_sync(0xffffffffu, n_vert, d);
        n_iso += __shfl_down_sync(0xffffffffu, n_iso, d);
        n_phantom += __shfl_down_sync(0xffffffffu, n_phantom, d);
    }
    if ((tid & 31) == 0) {
        if (n_vert) atomicAdd(&B.vertices, (unsigned long long)n_vert);
        if (n_iso) atomicAdd(&B.isolated, (unsigned long long)n_iso);
        if (n_phantom) atomicAdd(&B.phantom, (unsigned long long)n_phantom);
    }
    tsync<MODE>();

    clk[2] = clock64();
    // ---------------- W2: paths, walked from their ends ----------------
    // its list: the path ends W1 found, else a compaction (bottom of wl)
    const uint32_t n_ends = *(volatile uint32_t*)&B.end_n;
    const bool ends_listed = LISTS && n_ends <= cap_end;
    const bool ends_top = ends_listed && !l1_top;
    if (!ends_listed) {
        __syncthreads();   // every thread has read the count
        if (tid == 0) B.end_n = 0;
        __syncthreads();
        compact(per, wl, &B.end_n, [&](uint32_t ls) {
            if (local_empty<W>(lkeys, ls)) return false;
            const uint32_t m = lmeta[ls];
            return !(m & M_ISO) && (term_of(m, FRONT) != T_OK || term_of(m, BACK) != T_OK);
        });
        __syncthreads();
    }
    const uint32_t nw2 = ends_listed ? n_ends : *(volatile uint32_t*)&B.end_n;
    uint32_t n_cov = 0;   // vertices of what this thread emitted
    for (uint32_t base = 0; base < nw2; base += nt) {   // uniform over the CTA: warps reserve output together
        const uint32_t i = base + tid;
        // what this lane emits: one-k-mer cycles at s and/or e, and one path vs..ve
        bool kc0 = false, kc1 = false, mark0 = false, mark1 = false, path = false, lm = false;
        uint32_t s = 0, e = 0, n2 = 0, walked = 0;   // walked: vertices of the two-end walk (0: one vertex)
        unsigned long long steps0 = 0, steps1 = 0;   // bases of walk steps 1..32, 33..64
        Kmer<W> first{};
        DV<W> vs{}, ve{};
        int sd0 = BACK;
        EndInfo st{0, 0, true}, en{0, 0, true};
        bool best_canon = true;
        if (i < nw2) {
            const uint32_t ls = wl[ends_top ? per - 1 - i : i];
            s = base_slot + ls;
            e = s;
            const uint32_t meta = lmeta[ls];
            const bool okf = term_of(meta, FRONT) == T_OK, okb = term_of(meta, BACK) == T_OK;
            if (!okf && !okb) {         // one-vertex path
                if (looped_homopolymer(ops, T.key(s), st_ef(lst[sti<W>(ls)]), fth)) kc0 = true;
                else {
                    vs = dv_at(T, ops, s, BACK); ve = vs; sd0 = BACK; n2 = 1; path = true;
                    st = EndInfo{s, term_of(meta, FRONT), true}; en = EndInfo{s, term_of(meta, BACK), true};
                }
                lmeta[ls] = lmeta[ls] | M_VISITED;
            } else {
                const int side0 = okf ? FRONT : BACK;   // walk through the linked side
                const uint32_t ins0 = st_ins(lst[sti<W>(ls)]);
                const DV<W> v0 = dv_at(T, ops, s, side0);
                // pass 1: the other end, first-occurrence minima; the walk marks its vertices
                // and keeps the bases it steps through (2 bits each, up to STEP_BUF of them),
                // so the emitting end writes its label without walking again
                DV<W> v = v0; int side = side0;
                uint32_t n = 1;
                uint32_t v1_slot = s; int v1_side = side0;     // second vertex
                uint32_t vp_slot = s; int vp_side = side0;     // vertex before the current one
                uint32_t m_int = 0xffffffffu; bool m_int_canon = true;
                uint32_t cur_meta = meta;
                bool ok = true;
                T.or_meta(s, M_VISITED);
                while (term_of(cur_meta, side) == T_OK) {
                    if (n > 1) {   // v is interior
                        const uint32_t ic = st_ins(v.st);
                        if (ic < m_int) { m_int = ic; m_int_canon = side == BACK; }
                    }
                    vp_slot = v.slot; vp_side = side;
                    int s_in;
                    uint32_t b;   // the base the step appends in walk direction
                    if (links) {  // the neighbour W1 found: no lookup; v.d / v.r are rebuilt at the end
                        const uint32_t f = side_field(cur_meta, side);
                        const uint32_t e = ef_edge_at(st_ef(v.st), side, fth);
                        b = side == BACK ? e : 3 - e;
                        v.slot = (f >> 1) & (LINK_SLOTS - 1);
                        s_in = (int)(f >> 13);
                        v.st = T.ld_st(v.slot);
                    } else {
                        if (!step(T, ops, fth, v, side, s_in)) { atomicOr(a.err, DERR_MISSING_KEY); ok = false; break; }
                        b = ops.last_base(v.d);
                    }
                    side = 1 - s_in;
                    cur_meta = T.ld_meta(v.slot);
                    T.or_meta(v.slot, M_VISITED);
                    if (n <= STEP_BUF) {
                        const unsigned long long bb = (unsigned long long)b << (2 * ((n - 1) & 31));
                        if (n <= 32) steps0 |= bb; else steps1 |= bb;
                    }
                    if (n == 1) { v1_slot = v.slot; v1_side = side; }
                    if (++n > T.per * T.nranks + 1) { atomicOr(a.err, DERR_WALK_LIMIT); ok = false; break; }
                }
                if (links && ok && n > 1) v = dv_at(T, ops, v.slot, side);   // the end, leaving by `side`
                if (ok && v.slot >= s) {   // the end with the smaller slot emits
                    e = v.slot;
                    const int e_side = side;   // the walk stops at e's side e_side
                    const uint32_t meta_e = cur_meta;
                    const uint32_t ins1 = st_ins(v.st);
                    const bool q0 = looped_homopolymer(ops, side0 == BACK ? v0.d : v0.r, st_ef(v0.st), fth);
                    const bool q1 = looped_homopolymer(ops, side == BACK ? v.d : v.r, st_ef(v.st), fth);
                    uint32_t m = m_int;
                    if (!q0 && ins0 < m) m = ins0;
                    if (!q1 && ins1 < m) m = ins1;
                    const bool fake0 = q0 && ins0 < m, fake1 = q1 && ins1 < m;
                    kc0 = mark0 = fake0; kc1 = mark1 = fake1;
                    n2 = n - fake0 - fake1;
                    walked = n;
                    first = v0.d;
                    if (n2 > 0) {
                        path = true;
                        if (!fake0) { st = EndInfo{s, term_of(meta, 1 - side0), side0 == BACK}; vs = v0; sd0 = side0; }
                        else { st = EndInfo{v1_slot, T_CROSSED, v1_side == BACK}; vs = dv_at(T, ops, v1_slot, v1_side); sd0 = v1_side; }
                        if (!fake1) { en = EndInfo{e, term_of(meta_e, e_side), e_side == BACK}; ve = v; }
                        else { en = EndInfo{vp_slot, T_CROSSED, vp_side == BACK}; ve = dv_at(T, ops, vp_slot, vp_side); }
                        // first-inserted vertex of the emitted path and its orientation along the walk
                        uint32_t best = m_int; best_canon = m_int_canon;
                        if (!fake0 && ins0 < best) { best = ins0; best_canon = side0 == BACK; }
                        if (!fake1 && ins1 < best) { best = ins1; best_canon = e_side == BACK; }
                    }
                }
            }
            if (path) lm = st.term == T_EXIT || en.term == T_EXIT;
        }
        const uint32_t L = path ? n2 + k - 1 : 0;
        __syncwarp();
        const Res r = reserve_block(B.sk, B, (kc0 ? k + 4 : 0) + (kc1 ? k + 4 : 0) + (path && !lm ? L + 4 : 0),
                                   path && lm ? 1u : 0u, path && lm ? L : 0u);
        unsigned long long fo = r.fa;
        if (kc0) { write_kmer_cycle(T, ops, s, B, fo); fo += k + 4; }
        if (kc1) { write_kmer_cycle(T, ops, e, B, fo); fo += k + 4; }
        if (path) {
            const bool buffered = W <= 2 && walked > 0 && walked - 1 <= STEP_BUF;
            write_emitted_path(a, T, ops, vs, sd0, n2, ve, st, en, best_canon, B, lm, fo, r.lm_idx, r.lm_off,
                               buffered, steps0, steps1, first, kc0 ? 1u : 0u, links);
        }
        if (mark0) T.or_meta(s, M_VISITED);
        if (mark1) T.or_meta(e, M_VISITED);
        n_cov += (kc0 ? 1u : 0u) + (kc1 ? 1u : 0u) + (path ? n2 : 0u);
    }
    for (int d = 16; d; d >>= 1) n_cov += __shfl_down_sync(0xffffffffu, n_cov, d);
    if ((tid & 31) == 0 && n_cov) atomicAdd(&B.covered, n_cov);
    tsync<MODE>();

    clk[3] = clock64();
    // ---------------- W3: isolated cycles ----------------
    // Every path is emitted once, with its vertices counted: when they cover every vertex
    // with an edge, no isolated cycle is left (one CTA's table; a cluster's paths span CTAs)
    const bool no_cycles = MODE != CLUSTER && B.covered == B.vertices - B.isolated;
    if (!no_cycles) {
        compact(per, wl, &B.cyc_n, [&](uint32_t ls) {
            return !local_empty<W>(lkeys, ls) && !(lmeta[ls] & (M_ISO | M_VISITED));
        });
        __syncthreads();
        const uint32_t nw3 = B.cyc_n;
        for (uint32_t base = 0; base < nw3; base += nt) {
            const uint32_t i = base + tid;
            bool emit = false;
            uint32_t n = 0;
            DV<W> v0{};
            if (i < nw3) {
                const uint32_t ls = wl[i];
                const uint32_t s = base_slot + ls;
                if (!(*(volatile uint32_t*)(lmeta + ls) & M_VISITED)) {
                    // every vertex left has both sides linked: walk the cycle from s out of its back side
                    v0 = dv_at(T, ops, s, BACK);
                    DV<W> v = v0; int side = BACK;
                    bool is_min = true, ok = true;
                    do {
                        int s_in;
                        if (!step(T, ops, fth, v, side, s_in) || ++n > T.per * T.nranks) { atomicOr(a.err, DERR_WALK_LIMIT); ok = false; break; }
                        side = 1 - s_in;
                        if (v.slot != s && (v.d < v.r ? v.d : v.r) < v0.d) is_min = false;
                    } while (v.slot != s);
                    emit = ok && is_min;
                }
            }
            __syncwarp();
            const Res r = reserve_warp(B.sk, emit ? n + k + 3 : 0, 0, 0);
            if (emit) {
                // Character_Buffer::rotate_append_cycle (include/Character_Buffer.hpp:166-175): start at the
                // minimum vertex in its canonical orientation
                char* p = fasta_at(B.sk, r.fa, n + k - 1);
                write_path(T, ops, fth, v0, BACK, n, p, false, true, links);
                atomicAdd(&B.trivial, 1ull); atomicAdd(&B.icc, 1ull);
            }
        }
    }
    tsync<MODE>();
    clk[4] = clock64();

    if (a.dump) {
        for (uint32_t ls = tid; ls < per; ls += nt) {
            const uint32_t s = base_slot + ls;
            if (local_empty<W>(lkeys, ls)) continue;
            const unsigned long long i = atomicAdd(&a.cnt->dump_count, 1ull);
            if (i >= a.dump_cap) { atomicOr(a.err, DERR_DUMP_OVERFLOW); continue; }
            StateOut o;
            put_key(o.key, T.key(s));
            o.ef = st_ef(lst[sti<W>(ls)]); o.g = (uint16_t)B.sk.g; o.status = (uint8_t)(lmeta[ls] & 7); o.pad = 0;
            a.dump[i] = o;
        }
    }
    __syncthreads();
    if (tid == 0) {
        clk[5] = clock64();
        if (a.record_clocks)
            for (int i = 0; i < 5; ++i) atomicAdd(&a.cnt->phase_cycles[i], (unsigned long long)(clk[i + 1] - clk[i]));
        const unsigned long long v[6] = {B.vertices, B.isolated, B.phantom, B.trivial, B.icc, B.lmtig};
        if (a.bucket_cnt) {   // batch: per-subgraph counters, summed per job afterwards (no contended atomics)
            for (int i = 0; i < 5; ++i)
                if (v[i]) atomicAdd(a.bucket_cnt + 5ull * g + i, (uint32_t)v[i]);
        } else {
            for (int i = 0; i < 6; ++i)
                if (v[i]) atomicAdd(B.sk.cnt + i, v[i]);
        }
    }
    tsync<MODE>();   // no CTA leaves while another may still read its shared memory
}

template <int W>
__device__ __forceinline__ void carve(unsigned char* base, uint32_t per, unsigned long long*& keys, unsigned long long*& st,
                                      uint32_t*& meta, uint32_t*& wl) {
    constexpr size_t KB = W <= 2 ? 16 : 32;   // key bytes per slot
    keys = (unsigned long long*)base;
    st = W == 1 ? keys + 1 : (unsigned long long*)(base + (size_t)per * KB);   // k <= 31: interleaved with the keys
    meta = (uint32_t*)(base + (size_t)per * (W == 1 ? 16 : KB + 8));
    wl = meta + per;
}

// One subgraph per CTA (per = the table's whole capacity) or per cluster.  LB: the
// largest CTA.  k > 32 (104 registers at LB 512) has a second form for tables of up to
// 2048 slots, LB 256 at three CTAs per SM (80 registers): a 512-thread CTA of the wide
// form holds a whole SM's registers, so one subgraph's phase barriers idle the SM.
// k > 63 runs 256-thread CTAs, two per SM (128 registers).
constexpr int shared_min_blocks(int W, int LB) { return W > 2 ? 2 : LB <= 256 ? 3 : 1; }
template <int W, int MODE, int LB>
__global__ void __launch_bounds__(LB, shared_min_blocks(W, LB)) k_subgraph_shared(const SubgraphArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Block B;
    uint32_t rank = 0, nranks = 1;
    if constexpr (MODE == CLUSTER) { rank = cg::this_cluster().block_rank(); nranks = cg::this_cluster().num_blocks(); }
    const uint32_t per = a.smem_cap;
    Tab<W, MODE> T;
    unsigned long long *lk, *ls; uint32_t *lm, *wl;
    carve<W>(smem, per, lk, ls, lm, wl);
    T.keys = smem_addr(lk); T.st = smem_addr(ls); T.meta = smem_addr(lm); T.err_flag = a.err;
    T.per = per; T.nranks = nranks; T.rank = rank;
    T.shift = 31 - __clz(per); T.pmask = per - 1;
    Block* Bc = &B;
    if constexpr (MODE == CLUSTER) Bc = cg::this_cluster().map_shared_rank(&B, 0);
    // one pass over the list (grid = list x cluster), or a persistent grid striding through it
    const uint32_t* list = a.list + (a.list_base ? *a.list_base : 0u);
    const uint32_t n = a.list_n ? *a.list_n : a.n_list;
    for (uint32_t i = blockIdx.x / nranks; i < n; i += gridDim.x / nranks)
        run_subgraph<W, MODE>(a, T, B, Bc, list[i], rank, nranks, per, lk, ls, lm, wl);
}

// Tables in the arena: no shared memory to share, so k > 32 runs three 256-thread CTAs
// per SM (80 registers) instead of one of 512.
template <int W> struct GlobalBounds { static constexpr int threads = 512, min_blocks = 2; };   // 64 registers
template <> struct GlobalBounds<2> { static constexpr int threads = 256, min_blocks = 3; };     // 80 registers
template <> struct GlobalBounds<3> { static constexpr int threads = 256, min_blocks = 2; };     // 128 registers
template <> struct GlobalBounds<4> { static constexpr int threads = 256, min_blocks = 2; };
template <int W>
__global__ void __launch_bounds__(GlobalBounds<W>::threads, GlobalBounds<W>::min_blocks) k_subgraph_global(const SubgraphArgs a) {
    __shared__ Block B;
    const uint32_t lb = a.list_base ? *a.list_base : 0u;
    const uint32_t n = a.list_n ? *a.list_n : a.n_list;
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint32_t cap = a.tab_cap[lb + i];
        if (cap == 0) continue;   // no arena room: the job is redone on its own
        unsigned char* base = a.arena + a.tab_off[lb + i] * (uint64_t)slot_bytes(W);
        Tab<W, GLOBAL> T;
        unsigned long long *lk, *ls; uint32_t *lm, *wl;
        carve<W>(base, cap, lk, ls, lm, wl);
        T.keys = (uint64_t)lk; T.st = (uint64_t)ls; T.meta = (uint64_t)lm;
        T.per = cap; T.nranks = 1; T.rank = 0; T.shift = 31; T.pmask = 0xffffffffu; T.err_flag = a.err;
        run_subgraph<W, GLOBAL>(a, T, B, &B, a.list[lb + i], 0, 1, cap, lk, ls, lm, wl);
        __syncthreads();
    }
}

// The kernels' shared-memory limit is always raised to the largest table any launch
// uses (it is process-wide state: lowering it would break launches recorded in graphs).
template <int W> constexpr size_t max_table_bytes() { return (size_t)(W == 1 ? 8192 : W == 2 ? 4096 : 2048) * slot_bytes(W); }
template <typename K>
cudaError_t raise_smem_limit(K kernel, size_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// grid 0: one pass (list x cluster CTAs), which first raises the kernel's shared-memory
// limit; a persistent grid relies on subgraph_occupancy having raised it (no attribute
// calls while a stream is being captured).
template <typename K>
cudaError_t launch_shared(K kernel, const SubgraphArgs& a, uint32_t cluster, uint32_t threads, size_t bytes, cudaStream_t s,
                          uint32_t grid = 0, size_t limit = 0) {
    if (!grid) {
        cudaError_t e = raise_smem_limit(kernel, limit > bytes ? limit : bytes);
        if (e != cudaSuccess) return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid ? grid : a.n_list * cluster);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = cluster > 1 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, a);
}

}  // namespace

template <typename K>
int occupancy_of(K kernel, uint32_t cluster, uint32_t threads, size_t bytes, size_t limit) {
    if (raise_smem_limit(kernel, limit > bytes ? limit : bytes) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cluster <= 1) {
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, (int)threads, bytes) != cudaSuccess) { cudaGetLastError(); return 0; }
        return n;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kernel, &cfg) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

__global__ void k_stripe_fixup(LmtigOut* lm, uint64_t lm_slice, const unsigned long long* __restrict__ lm_used,
                               const unsigned long long* __restrict__ text_base, uint32_t stripes) {
    for (uint32_t st = blockIdx.y; st < stripes; st += gridDim.y) {
        const unsigned long long n = lm_used[st * JOB_CUR_STRIDE + 2];
        const unsigned long long base = text_base[st];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n && i < lm_slice; i += (uint64_t)gridDim.x * blockDim.x)
            lm[st * lm_slice + i].label_off += base;
    }
}

uint32_t subgraph_max_per_cta(int words) { return words == 1 ? 8192 : words == 2 ? 4096 : 2048; }
uint32_t subgraph_max_threads(int words, uint32_t per) {
    if (words > 2) return 256;                            // k > 63: one 256-thread form
    if (per == 0) return words == 1 ? 512 : 256;          // arena tables
    if (words == 1) return per > 4096 ? 1024 : 512;
    return per > 2048 ? 512 : 256;
}
uint32_t subgraph_cluster_per_cta(int words) { return words == 1 ? 4096 : 2048; }

namespace {
// the kernel of a one-CTA shared-memory table, by key words and CTA size
template <int W> cudaError_t launch_local_w(const SubgraphArgs& a, uint32_t threads, size_t bytes, cudaStream_t s,
                                            uint32_t grid, size_t limit) {
    if constexpr (W == 1) return launch_shared(k_subgraph_shared<1, LOCAL, 1024>, a, 1, threads, bytes, s, grid, limit);
    else if constexpr (W == 2)
        return threads <= 256 ? launch_shared(k_subgraph_shared<2, LOCAL, 256>, a, 1, threads, bytes, s, grid, limit)
                              : launch_shared(k_subgraph_shared<2, LOCAL, 512>, a, 1, threads, bytes, s, grid, limit);
    else return launch_shared(k_subgraph_shared<W, LOCAL, 256>, a, 1, threads, bytes, s, grid, limit);
}
template <int W> int occupancy_local_w(uint32_t threads, size_t bytes) {
    if constexpr (W == 1) return occupancy_of(k_subgraph_shared<1, LOCAL, 1024>, 1, threads, bytes, max_table_bytes<1>());
    else if constexpr (W == 2)
        return threads <= 256 ? occupancy_of(k_subgraph_shared<2, LOCAL, 256>, 1, threads, bytes, max_table_bytes<2>())
                              : occupancy_of(k_subgraph_shared<2, LOCAL, 512>, 1, threads, bytes, max_table_bytes<2>());
    else return occupancy_of(k_subgraph_shared<W, LOCAL, 256>, 1, threads, bytes, max_table_bytes<W>());
}
cudaError_t launch_local(const SubgraphArgs& a, int words, uint32_t threads, size_t bytes, cudaStream_t s, uint32_t grid) {
    switch (words) {
        case 1: return launch_local_w<1>(a, threads, bytes, s, grid, grid ? 0 : max_table_bytes<1>());
        case 2: return launch_local_w<2>(a, threads, bytes, s, grid, grid ? 0 : max_table_bytes<2>());
        case 3: return launch_local_w<3>(a, threads, bytes, s, grid, grid ? 0 : max_table_bytes<3>());
        case 4: return launch_local_w<4>(a, threads, bytes, s, grid, grid ? 0 : max_table_bytes<4>());
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t launch_global(const SubgraphArgs& a, int words, uint32_t threads, uint32_t grid, cudaStream_t s) {
    switch (words) {
        case 1: k_subgraph_global<1><<<grid, threads, 0, s>>>(a); break;
        case 2: k_subgraph_global<2><<<grid, threads, 0, s>>>(a); break;
        case 3: k_subgraph_global<3><<<grid, threads, 0, s>>>(a); break;
        case 4: k_subgraph_global<4><<<grid, threads, 0, s>>>(a); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_subgraphs(const SubgraphArgs& a, int words, uint32_t cluster, uint32_t threads, cudaStream_t s) {
    if (a.n_list == 0) return cudaSuccess;
    if (cluster == 0) {   // global-memory tables
        if (threads > subgraph_max_threads(words, 0)) return cudaErrorInvalidValue;
        return launch_global(a, words, threads, a.n_list, s);
    }
    const size_t bytes = (size_t)a.smem_cap * slot_bytes(words);
    if (threads > subgraph_max_threads(words, a.smem_cap)) return cudaErrorInvalidValue;
    if (cluster == 1) return launch_local(a, words, threads, bytes, s, 0);
    if (words != 1) return cudaErrorInvalidValue;   // k > 32 tables are one CTA's or the arena's
    return launch_shared(k_subgraph_shared<1, CLUSTER, 1024>, a, cluster, threads, bytes, s, 0, max_table_bytes<1>());
}

void launch_stripe_fixup(LmtigOut* lm, uint64_t lm_slice, const unsigned long long* lm_used,
                         const unsigned long long* text_base, uint32_t stripes, cudaStream_t s) {
    k_stripe_fixup<<<dim3(64, stripes), 256, 0, s>>>(lm, lm_slice, lm_used, text_base, stripes);
}

int subgraph_occupancy(int words, uint32_t cluster, uint32_t threads, uint32_t per) {
    const size_t bytes = (size_t)per * slot_bytes(words);
    if (threads > subgraph_max_threads(words, per)) return 0;
    if (cluster <= 1) {
        switch (words) {
            case 1: return occupancy_local_w<1>(threads, bytes);
            case 2: return occupancy_local_w<2>(threads, bytes);
            case 3: return occupancy_local_w<3>(threads, bytes);
            case 4: return occupancy_local_w<4>(threads, bytes);
            default: return 0;
        }
    }
    if (words != 1) return 0;   // no cluster tables for k > 32
    return occupancy_of(k_subgraph_shared<1, CLUSTER, 1024>, cluster, threads, bytes, max_table_bytes<1>());
}

cudaError_t launch_subgraphs_persistent(const SubgraphArgs& a, int words, uint32_t cluster, uint32_t threads,
                                        uint32_t per, uint32_t grid, cudaStream_t s) {
    if (grid == 0) return cudaSuccess;
    if (cluster == 0) {
        if (threads > subgraph_max_threads(words, 0)) return cudaErrorInvalidValue;
        return launch_global(a, words, threads, grid, s);
    }
    SubgraphArgs b = a;
    b.smem_cap = per;
    const size_t bytes = (size_t)per * slot_bytes(words);
    if (threads > subgraph_max_threads(words, per)) return cudaErrorInvalidValue;
    if (cluster == 1) return launch_local(b, words, threads, bytes, s, grid);
    if (words != 1) return cudaErrorInvalidValue;   // no cluster tables for k > 32
    return launch_shared(k_subgraph_shared<1, CLUSTER, 1024>, b, cluster, threads, bytes, s, grid);
}

}  // namespace cfg
