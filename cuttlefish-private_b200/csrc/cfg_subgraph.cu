// cfg_subgraph.cu -- K2 + K3: per-subgraph vertex table and local unitig walk.
//
// One CTA owns one subgraph.  Its open-addressing table lives in shared memory
// when it fits (global-memory arena otherwise) and holds per vertex: the
// canonical k-mer, the packed 4-bit edge frequencies and discontinuity flags of
// State_Config<false> (include/State_Config.hpp:24-268), and the stream position
// of the vertex's first occurrence.
//
// Build (Subgraph::construct, src/Subgraph.cpp:43-108): a thread per weak super
// k-mer rolls its k-mers and applies HT_Router::update (include/Subgraph.hpp:546-560)
// with CAS-updated saturating counters; the self-loop rule (:82-83) needs only the
// previous k-mer of the same super k-mer.
//
// Walk (Subgraph::contract / extract_maximal_unitig / walk_unitig,
// src/Subgraph.cpp:183-271, include/Subgraph.hpp:414-543): a step v -(side s)-> u
// is taken iff s holds one passing edge, u != v, and u's entrance side holds at
// most one.  That relation is symmetric, so the reference's sequential walk from
// any seed returns the whole maximal path, whatever the seed order, except in one
// case: a homopolymer vertex b^k whose back side holds only its own self-loop and
// whose front side holds at most one edge.  Seeded directly, the reference
// records it as a one-vertex cycle; reached from its predecessor, it ends that
// predecessor's unitig.  The reference seeds in table-insertion order (first
// occurrence), so the kernel compares first-occurrence positions to decide, and
// orients each lm-tig by its first-inserted vertex exactly as the reference does.
// Paths are walked from both ends in parallel; the end with the smaller slot emits.
#include "cfg_device.cuh"
#include "cfg_internal.h"

namespace cfg {

namespace {

constexpr uint32_t NONE = 0xffffffffu;
constexpr uint64_t EMPTY = ~0ull;
// walk termination kinds (Walk_Termination, include/Subgraph.hpp:362-369)
constexpr uint32_t T_OK = 0, T_BRANCHED = 1, T_CROSSED = 2, T_DEAD = 3, T_EXIT = 4;
// meta layout: bits 0-2 visited / disc front / disc back; 3 Q (self-looped homopolymer);
// 4 isolated; 8-10 front termination; 11-13 back termination
constexpr uint32_t M_Q = 8u, M_ISO = 16u;

__device__ __forceinline__ uint32_t term_of(uint32_t meta, int side) { return (meta >> (side == FRONT ? 8 : 11)) & 7; }
__device__ __forceinline__ uint32_t compb(uint32_t b) { return b < 4 ? 3 - b : b; }

template <int W, bool SM>
struct Tab {
    unsigned long long* keys;   // W words per slot
    uint32_t* ef;
    uint32_t* meta;
    uint32_t* ins;
    uint32_t* nbr;              // 2 per slot: (slot << 1 | entrance side) or NONE
    uint32_t mask;

    template <typename T> __device__ __forceinline__ T ld(const T* p) const {
        if constexpr (SM) return *(const volatile T*)p;
        else return __ldcg(p);
    }
    __device__ __forceinline__ Kmer<W> key(uint32_t s) const {
        if constexpr (W == 1) return Kmer<1>{ld(keys + s)};
        else return Kmer<2>{ld(keys + 2 * s), ld(keys + 2 * s + 1)};
    }
    __device__ __forceinline__ bool empty(uint32_t s) const {
        if constexpr (W == 1) return ld(keys + s) == EMPTY;
        else return ld(keys + 2 * s + 1) == EMPTY;
    }
    __device__ uint32_t find(const Kmer<W>& x) const {   // read-only phase
        uint32_t h = (uint32_t)key_hash(x) & mask;
        for (uint32_t p = 0; p <= mask; ++p) {
            if (empty(h)) return NONE;
            if (key(h) == x) return h;
            h = (h + 1) & mask;
        }
        return NONE;
    }
    __device__ uint32_t find_or_insert(const Kmer<W>& x, bool& fresh) {
        uint32_t h = (uint32_t)key_hash(x) & mask;
        fresh = false;
        for (uint32_t p = 0; p <= mask; ++p) {
            if constexpr (W == 1) {
                const unsigned long long cur = ld(keys + h);
                if (cur == x.lo) return h;
                if (cur == EMPTY) {
                    const unsigned long long old = atomicCAS(keys + h, EMPTY, (unsigned long long)x.lo);
                    if (old == EMPTY) { fresh = true; return h; }
                    if (old == x.lo) return h;
                }
            } else {
                const unsigned long long hi = ld(keys + 2 * h + 1);
                if (hi == EMPTY || hi == x.hi) {
                    uint64_t olo, ohi;
                    cas128(keys + 2 * h, EMPTY, EMPTY, x.lo, x.hi, olo, ohi);
                    if (olo == EMPTY && ohi == EMPTY) { fresh = true; return h; }
                    if (olo == x.lo && ohi == x.hi) return h;
                }
            }
            h = (h + 1) & mask;
        }
        return NONE;
    }
};

struct Block {   // per-CTA shared bookkeeping
    uint32_t inserted, overflow;
    unsigned long long vertices, isolated, phantom, trivial, icc, lmtig;
};

template <int W>
__device__ __forceinline__ Kmer<W> phi_kmer(const KOps<W>& ops) {   // all-T k-mer, include/Discontinuity_Graph.hpp:44-49
    Kmer<W> x;
    if constexpr (W == 1) x.lo = ops.mask;
    else { x.lo = ~0ull; x.hi = ops.mhi; }
    return x;
}

template <int W>
__device__ __forceinline__ void put_key(uint64_t out[2], const Kmer<W>& x) {
    out[0] = x.lo;
    out[1] = x.hi_word();
}

// Writes the label of the path that starts at (slot, exit side) and has n vertices.
template <int W, bool SM>
__device__ void write_path(const Tab<W, SM>& T, const KOps<W>& ops, uint32_t s0, int side0, uint32_t n, char* dst, bool rev) {
    const uint32_t k = ops.k;
    const uint32_t L = n + k - 1;
    const Kmer<W> x = T.key(s0);
    const Kmer<W> d = side0 == BACK ? x : ops.rc(x);
    auto put = [&](uint32_t i, uint32_t b) {
        if (!rev) dst[i] = "ACGT"[b];
        else dst[L - 1 - i] = "ACGT"[3 - b];
    };
    for (uint32_t i = 0; i < k; ++i) put(i, ops.base(d, i));
    uint32_t cur = s0; int side = side0;
    for (uint32_t t = 1; t < n; ++t) {
        const uint32_t nb = T.ld(T.nbr + 2 * cur + side);
        const uint32_t u = nb >> 1; const int s_in = (int)(nb & 1);
        const Kmer<W> ku = T.key(u);
        put(k - 1 + t, s_in == FRONT ? ops.last_base(ku) : 3 - ops.first_base(ku));
        cur = u; side = 1 - s_in;
    }
}

template <int W>
__device__ __forceinline__ char* reserve_fasta(const SubgraphArgs& a, uint32_t L) {
    const unsigned long long off = atomicAdd(&a.cnt->fasta_bytes, (unsigned long long)(L + 4));
    if (off + L + 4 > a.fasta_cap) { atomicOr(a.err, DERR_OUT_OVERFLOW); return nullptr; }
    char* p = a.fasta + off;
    p[0] = '>'; p[1] = '0'; p[2] = '\n'; p[3 + L] = '\n';
    return p + 3;
}

template <int W, bool SM>
__device__ void emit_kmer_cycle(const SubgraphArgs& a, const Tab<W, SM>& T, const KOps<W>& ops, uint32_t s, Block& B) {
    char* p = reserve_fasta<W>(a, ops.k);
    if (p) { const Kmer<W> x = T.key(s); for (uint32_t i = 0; i < ops.k; ++i) p[i] = "ACGT"[ops.base(x, i)]; }
    atomicAdd(&B.trivial, 1ull); atomicAdd(&B.icc, 1ull);
}

struct EndInfo { uint32_t slot; uint32_t term; bool canon; };   // an end of a path in walk direction

template <int W, bool SM>
__device__ void emit_path(const SubgraphArgs& a, const Tab<W, SM>& T, const KOps<W>& ops, uint32_t g,
                          uint32_t s0, int side0, uint32_t n, EndInfo st, EndInfo en, bool seed_canon, Block& B) {
    const uint32_t k = ops.k;
    const uint32_t L = n + k - 1;
    const bool lm = st.term == T_EXIT || en.term == T_EXIT;
    if (!lm) {
        // trivial maximal unitig in canonical orientation (Maximal_Unitig_Scratch::finalize, :200-222)
        const Kmer<W> xs = T.key(st.slot), xe = T.key(en.slot);
        const Kmer<W> first = st.canon ? xs : ops.rc(xs);
        const Kmer<W> last_rc = en.canon ? ops.rc(xe) : xe;
        const bool rev = last_rc < first;
        char* p = reserve_fasta<W>(a, L);
        if (p) write_path(T, ops, s0, side0, n, p, rev);
        atomicAdd(&B.trivial, 1ull);
        return;
    }
    // lm-tig oriented by its first-inserted vertex (finalize_weak, :225-233; Unitig_File add, include/Unitig_File.hpp:338-359)
    const bool rev = !seed_canon;
    const EndInfo eu = rev ? en : st, ev = rev ? st : en;
    const bool u_first_canon = rev ? !en.canon : st.canon;     // label's first k-mer canonical?
    const bool v_last_canon = rev ? !st.canon : en.canon;      // label's last k-mer canonical?
    const unsigned long long idx = atomicAdd(&a.cnt->lm_count, 1ull);
    const unsigned long long off = atomicAdd(&a.cnt->lm_bytes, (unsigned long long)L);
    atomicAdd(&B.lmtig, 1ull);
    if (idx >= a.lm_cap || off + L > a.lm_text_cap) { atomicOr(a.err, DERR_OUT_OVERFLOW); return; }
    write_path(T, ops, s0, side0, n, a.lm_text + off, rev);
    LmtigOut o;
    const Kmer<W> phi = phi_kmer(ops);
    const bool u_exit = eu.term == T_EXIT, v_exit = ev.term == T_EXIT;
    put_key(o.u, u_exit ? T.key(eu.slot) : phi);
    put_key(o.v, v_exit ? T.key(ev.slot) : phi);
    const uint32_t s_u_back = u_exit ? (u_first_canon ? 1u : 0u) : 1u;
    const uint32_t s_v_back = v_exit ? (v_last_canon ? 0u : 1u) : 1u;
    o.label_off = off; o.label_len = L; o.g = (uint16_t)g;
    o.flags = (uint8_t)(s_u_back | (s_v_back << 1) | ((!u_exit) << 2) | ((!v_exit) << 3));
    o.pad = 0;
    a.lm[idx] = o;
}

template <int W, bool SM>
__device__ void run_subgraph(const SubgraphArgs& a, Tab<W, SM> T, uint32_t g, uint32_t cap, Block& B) {
    const KOps<W> ops(a.k);
    const uint32_t k = a.k, fth = a.fth;
    const uint32_t tid = threadIdx.x, nt = blockDim.x;

    for (uint32_t s = tid; s < cap; s += nt) {
        if constexpr (W == 1) T.keys[s] = EMPTY; else { T.keys[2 * s] = EMPTY; T.keys[2 * s + 1] = EMPTY; }
        T.ef[s] = 0; T.meta[s] = 0; T.ins[s] = 0xffffffffu;
    }
    if (tid == 0) { B.inserted = 0; B.overflow = 0; B.vertices = B.isolated = B.phantom = B.trivial = B.icc = B.lmtig = 0; }
    __syncthreads();

    // ---------------- build ----------------
    const uint32_t limit = (uint32_t)(((uint64_t)cap * a.load_limit_pct) / 100);
    const uint32_t r0 = a.bucket_off[g], r1 = a.bucket_off[g + 1];
    for (uint32_t r = r0 + tid; r < r1; r += nt) {
        if (*(volatile uint32_t*)&B.overflow) break;
        const uint64_t rec = a.recs[r];
        const uint32_t pos = rec_pos(rec), len = rec_len(rec), ld = rec_ld(rec), rd = rec_rd(rec);
        Kmer<W> fw = ops.load(a.packed, pos);
        Kmer<W> rc = ops.rc(fw);
        Kmer<W> pred_can = fw;
        for (uint32_t idx = 0;; ++idx) {
            const bool canon = fw < rc;
            const Kmer<W> can = canon ? fw : rc;
            const uint32_t pred = idx == 0 ? BASE_E : base_at(a.packed, pos + idx - 1);
            const uint32_t succ = idx + k == len ? BASE_E : base_at(a.packed, pos + idx + k);
            uint32_t front = canon ? pred : compb(succ);
            uint32_t back = canon ? succ : compb(pred);
            if (idx > 0 && can == pred_can) { if (canon) front = BASE_E; else back = BASE_E; }
            bool fresh;
            const uint32_t s = T.find_or_insert(can, fresh);
            if (s == NONE) { atomicOr(&B.overflow, 1u); break; }
            if (fresh && atomicAdd(&B.inserted, 1u) + 1 > limit) { atomicOr(&B.overflow, 1u); break; }
            uint32_t cur = T.ld(T.ef + s);
            for (uint32_t it = 0;; ++it) {
                const uint32_t nv = ef_add(cur, front, back);
                if (nv == cur) break;
                const uint32_t old = atomicCAS(T.ef + s, cur, nv);
                if (old == cur) break;
                cur = old;
                if (it > (1u << 22)) { atomicOr(a.err, DERR_CAS_LIMIT); break; }
            }
            const uint32_t p = pos + idx;
            if (p < T.ld(T.ins + s)) atomicMin(T.ins + s, p);
            uint32_t disc = 0;
            if (idx == 0 && ld) disc |= canon ? M_DISC_F : M_DISC_B;            // entrance side
            if (idx + k == len && rd) disc |= canon ? M_DISC_B : M_DISC_F;      // exit side
            if (disc && (T.ld(T.meta + s) & disc) != disc) atomicOr(T.meta + s, disc);
            if (idx + k == len) break;
            pred_can = can;
            ops.push_back(fw, succ);
            ops.push_front(rc, 3 - succ);
        }
    }
    __syncthreads();
    if (B.overflow) {
        if (tid == 0) {
            const unsigned long long i = atomicAdd(&a.cnt->retry_count, 1ull);
            a.retry[i] = g;
        }
        return;
    }

    // ---------------- W1: neighbour links ----------------
    for (uint32_t s = tid; s < cap; s += nt) {
        if (T.empty(s)) continue;
        const uint32_t ef = T.ef[s];
        uint32_t meta = T.meta[s];
        const uint32_t cf = ef_count(ef, FRONT, fth), cb = ef_count(ef, BACK, fth);
        atomicAdd(&B.vertices, 1ull);
        if (cf == 0 && cb == 0) {
            atomicAdd(&B.isolated, 1ull);
            if (meta & (M_DISC_F | M_DISC_B)) atomicAdd(&B.phantom, 1ull);
            T.meta[s] = meta | M_ISO;
            T.nbr[2 * s] = NONE; T.nbr[2 * s + 1] = NONE;
            continue;
        }
        const Kmer<W> x = T.key(s);
        const Kmer<W> xr = ops.rc(x);
        for (int side = 0; side < 2; ++side) {
            const uint32_t e = ef_edge_at(ef, side, fth);
            uint32_t term = T_OK, link = NONE;
            if (e == BASE_N) term = T_BRANCHED;
            else if (e == BASE_E) term = (meta & (side == FRONT ? M_DISC_F : M_DISC_B)) ? T_EXIT : T_DEAD;
            else {
                Kmer<W> y, yr;
                if (side == BACK) { y = x; ops.push_back(y, e); yr = xr; ops.push_front(yr, 3 - e); }
                else { y = xr; ops.push_back(y, 3 - e); yr = x; ops.push_front(yr, e); }
                const bool yc = y < yr;
                const uint32_t u = T.find(yc ? y : yr);
                const int s_in = yc ? FRONT : BACK;
                if (u == NONE) { atomicOr(a.err, DERR_MISSING_KEY); term = T_CROSSED; }
                else if (u == s) term = T_CROSSED;                               // self-loop
                else if (ef_count(T.ef[u], s_in, fth) > 1) term = T_CROSSED;     // branching entrance
                else link = (u << 1) | (uint32_t)s_in;
            }
            T.nbr[2 * s + side] = link;
            meta |= term << (side == FRONT ? 8 : 11);
        }
        // homopolymer b^k (b in {A, C}) whose back side holds only its self-loop
        const uint32_t eb = ef_edge_at(ef, BACK, fth);
        if (eb < 2 && cf <= 1 && ops.is_homopolymer(x, eb)) meta |= M_Q;
        T.meta[s] = meta;
    }
    __syncthreads();

    // ---------------- W2: paths, walked from their ends ----------------
    for (uint32_t s = tid; s < cap; s += nt) {
        if (T.empty(s)) continue;
        const uint32_t meta = T.meta[s];
        if (meta & M_ISO) continue;
        const uint32_t nf = T.nbr[2 * s], nb = T.nbr[2 * s + 1];
        if (nf != NONE && nb != NONE) continue;   // interior (or cycle) vertex
        if (nf == NONE && nb == NONE) {           // one-vertex path
            if (meta & M_Q) emit_kmer_cycle(a, T, ops, s, B);
            else {
                const EndInfo st{s, term_of(meta, FRONT), true}, en{s, term_of(meta, BACK), true};
                emit_path(a, T, ops, g, s, BACK, 1, st, en, true, B);
            }
            T.meta[s] = meta | M_VISITED;
            continue;
        }
        const int side0 = nf != NONE ? FRONT : BACK;   // walk through the linked side
        // pass 1: find the other end, first-occurrence minima
        uint32_t cur = s; int side = side0;
        uint32_t n = 1;
        uint32_t p1 = NONE; int p1_side = 0;          // second vertex
        uint32_t prev = NONE; int prev_side = 0;      // vertex before the current one
        uint32_t m_int = 0xffffffffu; bool m_int_canon = true;
        bool ok = true;
        while (true) {
            const uint32_t lnk = T.nbr[2 * cur + side];
            if (lnk == NONE) break;
            if (cur != s) {   // cur is interior
                const uint32_t ic = T.ins[cur];
                if (ic < m_int) { m_int = ic; m_int_canon = side == BACK; }
            }
            prev = cur; prev_side = side;
            cur = lnk >> 1; side = 1 - (int)(lnk & 1);
            if (n == 1) { p1 = cur; p1_side = side; }
            if (++n > cap + 1) { atomicOr(a.err, DERR_WALK_LIMIT); ok = false; break; }
        }
        if (!ok) continue;
        const uint32_t e = cur; const int e_side = side;   // other end, walk stops at its side e_side
        if (e < s) continue;                                // the smaller end emits
        const uint32_t meta_e = T.meta[e];
        const uint32_t ins0 = T.ins[s], ins1 = T.ins[e];
        const bool q0 = meta & M_Q, q1 = meta_e & M_Q;
        uint32_t m = m_int;
        if (!q0 && ins0 < m) m = ins0;
        if (!q1 && ins1 < m) m = ins1;
        const bool fake0 = q0 && ins0 < m, fake1 = q1 && ins1 < m;
        if (fake0) emit_kmer_cycle(a, T, ops, s, B);
        if (fake1) emit_kmer_cycle(a, T, ops, e, B);
        const uint32_t n2 = n - fake0 - fake1;
        if (n2 > 0) {
            EndInfo st, en;
            uint32_t s0; int sd0;
            if (!fake0) { st = EndInfo{s, term_of(meta, 1 - side0), side0 == BACK}; s0 = s; sd0 = side0; }
            else { st = EndInfo{p1, T_CROSSED, p1_side == BACK}; s0 = p1; sd0 = p1_side; }
            if (!fake1) en = EndInfo{e, term_of(meta_e, e_side), e_side == BACK};
            else en = EndInfo{prev, T_CROSSED, prev_side == BACK};
            // first-inserted vertex of the emitted path and its orientation along the walk
            uint32_t best = m_int; bool best_canon = m_int_canon;
            if (!fake0 && ins0 < best) { best = ins0; best_canon = side0 == BACK; }
            if (!fake1 && ins1 < best) { best = ins1; best_canon = e_side == BACK; }
            emit_path(a, T, ops, g, s0, sd0, n2, st, en, best_canon, B);
        }
        // mark the whole path visited
        cur = s; side = side0;
        T.meta[cur] |= M_VISITED;
        for (uint32_t t = 1; t < n; ++t) {
            const uint32_t lnk = T.nbr[2 * cur + side];
            cur = lnk >> 1; side = 1 - (int)(lnk & 1);
            T.meta[cur] |= M_VISITED;
        }
    }
    __syncthreads();

    // ---------------- W3: isolated cycles ----------------
    for (uint32_t s = tid; s < cap; s += nt) {
        if (T.empty(s)) continue;
        const uint32_t meta = T.ld(T.meta + s);
        if (meta & (M_ISO | M_VISITED)) continue;
        // every vertex left has both sides linked: walk the cycle from s out of its back side
        const Kmer<W> xs = T.key(s);
        uint32_t cur = s; int side = BACK; uint32_t n = 0;
        bool is_min = true, ok = true;
        do {
            const uint32_t lnk = T.nbr[2 * cur + side];
            if (lnk == NONE || ++n > cap) { atomicOr(a.err, DERR_WALK_LIMIT); ok = false; break; }
            cur = lnk >> 1; side = 1 - (int)(lnk & 1);
            if (cur != s && T.key(cur) < xs) is_min = false;
        } while (cur != s);
        if (!ok || !is_min) continue;
        // Character_Buffer::rotate_append_cycle (include/Character_Buffer.hpp:166-175): start at the
        // minimum vertex in its canonical orientation
        char* p = reserve_fasta<W>(a, n + k - 1);
        if (p) write_path(T, ops, s, BACK, n, p, false);
        atomicAdd(&B.trivial, 1ull); atomicAdd(&B.icc, 1ull);
        cur = s; side = BACK;
        for (uint32_t t = 0; t < n; ++t) {
            T.meta[cur] |= M_VISITED;
            const uint32_t lnk = T.nbr[2 * cur + side];
            cur = lnk >> 1; side = 1 - (int)(lnk & 1);
        }
    }
    __syncthreads();

    if (a.dump) {
        for (uint32_t s = tid; s < cap; s += nt) {
            if (T.empty(s)) continue;
            const unsigned long long i = atomicAdd(&a.cnt->dump_count, 1ull);
            if (i >= a.dump_cap) { atomicOr(a.err, DERR_DUMP_OVERFLOW); continue; }
            StateOut o;
            put_key(o.key, T.key(s));
            o.ef = T.ef[s]; o.g = (uint16_t)g; o.status = (uint8_t)(T.meta[s] & 7); o.pad = 0;
            a.dump[i] = o;
        }
    }
    if (tid == 0) {
        atomicAdd(&a.cnt->vertices, B.vertices); atomicAdd(&a.cnt->isolated, B.isolated);
        atomicAdd(&a.cnt->phantom, B.phantom); atomicAdd(&a.cnt->trivial, B.trivial);
        atomicAdd(&a.cnt->icc, B.icc); atomicAdd(&a.cnt->lmtig, B.lmtig);
    }
}

template <int W>
__global__ void __launch_bounds__(256) k_subgraph_smem(const SubgraphArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ Block B;
    const uint32_t cap = a.smem_cap;
    Tab<W, true> T;
    T.keys = (unsigned long long*)smem;
    T.ef = (uint32_t*)(smem + (size_t)cap * 8 * W);
    T.meta = T.ef + cap;
    T.ins = T.meta + cap;
    T.nbr = T.ins + cap;
    T.mask = cap - 1;
    for (uint32_t i = blockIdx.x; i < a.n_list; i += gridDim.x) {
        const uint32_t g = a.list[i];
        run_subgraph<W, true>(a, T, g, cap, B);
        __syncthreads();
    }
}

template <int W>
__global__ void __launch_bounds__(512) k_subgraph_global(const SubgraphArgs a) {
    __shared__ Block B;
    for (uint32_t i = blockIdx.x; i < a.n_list; i += gridDim.x) {
        const uint32_t g = a.list[i];
        const uint32_t cap = a.tab_cap[i];
        unsigned char* base = a.arena + a.tab_off[i] * (uint64_t)slot_bytes(W);
        Tab<W, false> T;
        T.keys = (unsigned long long*)base;
        T.ef = (uint32_t*)(base + (size_t)cap * 8 * W);
        T.meta = T.ef + cap;
        T.ins = T.meta + cap;
        T.nbr = T.ins + cap;
        T.mask = cap - 1;
        run_subgraph<W, false>(a, T, g, cap, B);
        __syncthreads();
    }
}

}  // namespace

int subgraph_max_smem_cap(int words) { return words == 1 ? 4096 : 4096; }

void launch_subgraphs(const SubgraphArgs& a, int words, bool smem, uint32_t threads, cudaStream_t s) {
    if (a.n_list == 0) return;
    const unsigned grid = a.n_list;
    if (smem) {
        const size_t bytes = (size_t)a.smem_cap * slot_bytes(words);
        if (words == 1) {
            cudaFuncSetAttribute(k_subgraph_smem<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            k_subgraph_smem<1><<<grid, threads, bytes, s>>>(a);
        } else {
            cudaFuncSetAttribute(k_subgraph_smem<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            k_subgraph_smem<2><<<grid, threads, bytes, s>>>(a);
        }
    } else {
        if (words == 1) k_subgraph_global<1><<<grid, threads, 0, s>>>(a);
        else k_subgraph_global<2><<<grid, threads, 0, s>>>(a);
    }
}

}  // namespace cfg
