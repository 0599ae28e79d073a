// cfg_unitig.cu -- lm-tigs joined into maximal unitigs on the device.
//
// The discontinuity-graph phases of dBG_Contractor::construct
// (Discontinuity_Graph_Contractor::contract, Contracted_Graph_Expander::expand,
// Unitig_Collator::collate; src/dBG_Contractor.cpp:73-101) for an in-memory edge
// set, as data-parallel steps over the lm-tigs of one run:
//   1. pair the lm-tig ends that meet at a discontinuity vertex (a hash table on the
//      vertex k-mer; a vertex carries at most one lm-tig on each side);
//   2. list ranking over the 2n (lm-tig, direction) entries: each entry's predecessor
//      is the entry that leaves through its partner end, and every entry needs its
//      list's head and the label bases before it (each lm-tig adds its length minus
//      the k-base overlap).  Sparse ruling set (Reid-Miller's list ranking; the GPU
//      form of Rehman, Kothapalli & Narayanan, ICS 2009): heads, tails and a hashed
//      1/16 sample of the entries are splitters; from every splitter one thread walks
//      back to the previous splitter, labelling the entries it passes with their
//      distance to it; pointer jumping then ranks the splitters alone, and one pass
//      gives every entry its rank from its splitter's;
//   3. of the two mirror lists of a chain, take the one whose head end has the
//      smaller id (the host collator's walk), then flip it if its reverse complement
//      starts with a smaller k-mer (Maximal_Unitig::canonicalize,
//      include/Unitig_Collator.hpp:308-347);
//   4. reserve each unitig's FASTA record, and let every lm-tig copy its label (read
//      forward or reverse-complemented) to its offset -- all of it at the unitig's
//      tail, all but the last k bases elsewhere (its successor writes the k-mer they
//      share).
// Entries that never reach a head lie on closed chains (cycles): a second set of passes
// (collate_cycles_on_device, below) joins them and writes each cycle from its canonical
// start.
#include "cuttlefish_gpu.h"
#include "cfg_host.h"
#include "cfg_internal.h"

#include <algorithm>

namespace cfg {

namespace {

constexpr uint32_t NONE = 0xffffffffu;

// Vertex table slot: the first and the second lm-tig end seen at a vertex (NONE when
// free).  The vertex k-mer is not stored: it is read from the first end's lm-tig.
using EndSlot = uint2;

// One (lm-tig, direction) entry of the ranking: predecessor still to jump over (NONE
// once resolved), the farthest known ancestor (the head once resolved), and the label
// bases of the entries between them.
struct RankRec { uint32_t P, R; unsigned long long A; };

// Ranking marks: an entry that no splitter's walk passed lies on a closed chain.
constexpr uint32_t UNOWNED = 0xfffffffeu;
constexpr uint32_t SPLIT = 0x80000000u;    // node[x].y: x is a splitter (low bits: its id)
constexpr uint32_t OWNED = 0x80000000u;    // node[x].x: a walk passed x (low bits: its splitter)

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z ^= z >> 33; z *= 0xFF51AFD7ED558CCDull;
    z ^= z >> 33; z *= 0xC4CEB9FE1A85EC53ull;
    z ^= z >> 33;
    return z;
}


// An lm-tig end as the pairing pass reads it: the vertex k-mer's words with the end's side
// in bit 62 and its phi flag in bit 63 of the last word -- 16 bytes (words 0, 1) for
// k <= 63, 32 bytes (words 0..3) for k <= 127; the highest word of a k-mer leaves both
// bits free.  ew: 2 or 4 words per end.
constexpr unsigned long long END_SIDE = 1ull << 62, END_PHI = 1ull << 63;
__device__ __forceinline__ void put_ends(ulonglong2* ends, uint64_t g, const LmtigOut& m, uint32_t ew) {
    const unsigned long long fu = ((m.flags & 1ull) << 62) | ((m.flags >> 2 & 1ull) << 63);
    const unsigned long long fv = ((m.flags >> 1 & 1ull) << 62) | ((m.flags >> 3 & 1ull) << 63);
    if (ew == 2) {
        ends[2 * g] = make_ulonglong2(m.u[0], m.u[1] | fu);
        ends[2 * g + 1] = make_ulonglong2(m.v[0], m.v[1] | fv);
    } else {
        ends[4 * g] = make_ulonglong2(m.u[0], m.u[1]);
        ends[4 * g + 1] = make_ulonglong2(m.u[2], m.u[3] | fu);
        ends[4 * g + 2] = make_ulonglong2(m.v[0], m.v[1]);
        ends[4 * g + 3] = make_ulonglong2(m.v[2], m.v[3] | fv);
    }
}
// end e's k-mer words (flags cleared) and its flag word
template <int EW> struct EndKey {
    unsigned long long w[EW], flags;
    __device__ __forceinline__ EndKey(const ulonglong2* __restrict__ ends, uint64_t e) {
        if constexpr (EW == 2) {
            const ulonglong2 a = ends[e];
            w[0] = a.x; w[1] = a.y & ~(END_SIDE | END_PHI); flags = a.y;
        } else {
            const ulonglong2 a = ends[2 * e], b = ends[2 * e + 1];
            w[0] = a.x; w[1] = a.y; w[2] = b.x; w[3] = b.y & ~(END_SIDE | END_PHI); flags = b.y;
        }
    }
    __device__ __forceinline__ bool same(const EndKey& o) const {
        bool e = true;
#pragma unroll
        for (int j = 0; j < EW; ++j) e &= w[j] == o.w[j];
        return e;
    }
    __device__ __forceinline__ uint64_t hash() const {
        uint64_t h = mix64(w[EW - 1] + 0x9E3779B97F4A7C15ull);
#pragma unroll
        for (int j = EW - 2; j >= 1; --j) h = mix64(w[j] ^ h);
        return mix64(w[0] ^ h);
    }
};

// 0: gather the striped lm-tigs into one array with their label addresses.
__global__ void k_ut_gather(const LmtigOut* lm, uint64_t lm_slice, const char* text, uint64_t text_slice,
                            const unsigned long long* __restrict__ lm_base, const unsigned long long* __restrict__ text_base,
                            const unsigned long long* __restrict__ stripe_cur, uint32_t stripes,
                            const char** label, uint32_t* lens, ulonglong2* ends, uint32_t ew) {
    for (uint32_t st = blockIdx.y; st < stripes; st += gridDim.y) {
        const unsigned long long n = stripe_cur[st * JOB_CUR_STRIDE + 2];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
            const LmtigOut m = lm[st * lm_slice + i];
            const uint64_t g = lm_base[st] + i;
            lens[g] = m.label_len;
            put_ends(ends, g, m, ew);
            label[g] = text + st * text_slice + (m.label_off - text_base[st]);
        }
    }
}

// 0 (batch): gather every job's lm-tigs from its regions; the job rides along.
__global__ void k_ut_gather_jobs(const LmtigOut* lm, const char* text, const JobOut* __restrict__ jobs, uint32_t n_jobs,
                                 const unsigned long long* __restrict__ job_n, const unsigned long long* __restrict__ job_lm_base,
                                 const char** label, uint32_t* out_job, uint32_t* lens,
                                 ulonglong2* ends, uint32_t ew) {
    for (uint32_t j = blockIdx.y; j < n_jobs; j += gridDim.y) {
        const unsigned long long n = job_n[j];
        const JobOut& J = jobs[j];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
            const LmtigOut m = lm[J.lm_off + i];
            const uint64_t g = job_lm_base[j] + i;
            lens[g] = m.label_len;
            put_ends(ends, g, m, ew);
            label[g] = text + J.lm_text_off + m.label_off;
            out_job[g] = j;
        }
    }
}

// 1: every non-phi end into the vertex table; the second end at a vertex pairs with
// the first (a third end, or two ends on one side of the vertex, is an invalid graph).
// In a batch job j's ends have their own region of the table, [4 base_j, 4 (base_j +
// n_j)) -- its lm-tigs are [base_j, base_j + n_j) -- so a vertex is (job, k-mer) by
// construction.  Blocks take tiles of ends from a counter, in order, so the ends in
// flight span a window of about one job and the table slots, lm-tigs and partners
// they touch stay in L2 (one large job is inserted in one pass all the same: slicing
// its region to fit L2 re-reads every end per slice and measured slower).  The slot's
// first end is claimed by CAS and its k-mer read from the (immutable) lm-tig, so no
// thread waits on another.
constexpr uint32_t INSERT_TILE = 1024;
template <int EW>
__global__ void __launch_bounds__(256, 6) k_ut_insert(const ulonglong2* __restrict__ ends, const uint32_t* __restrict__ job,
                                                    uint64_t n, uint32_t* tab,
                                                    const unsigned long long* __restrict__ job_lm_base,
                                                    const unsigned long long* __restrict__ job_n,
                                                    unsigned long long* tiles, uint32_t* partner,
                                                    uint32_t* err) {
    __shared__ unsigned long long tile;
    const uint64_t n2 = 2 * n;
    for (;;) {
        if (threadIdx.x == 0) tile = atomicAdd(tiles, 1ull);
        __syncthreads();
        const uint64_t t0 = tile * INSERT_TILE;
        __syncthreads();
        if (t0 >= n2) return;
        for (uint32_t u = threadIdx.x; u < INSERT_TILE; u += blockDim.x) {
            const uint64_t e = t0 + u;
            if (e >= n2) break;
            const EndKey<EW> me(ends, e);
            if (me.flags & END_PHI) continue;
            const uint64_t h = me.hash();
            const uint32_t jb = job ? job[e >> 1] : 0u;
            const uint64_t base = job ? 4 * job_lm_base[jb] : 0, t = job ? 4 * job_n[jb] : 4 * n;
            uint64_t p = base + __umul64hi(h, t);
            for (uint64_t probe = 0; probe < t; ++probe) {
                const uint32_t old = atomicCAS(tab + 2 * p, NONE, (uint32_t)e);
                if (old == NONE) break;
                const EndKey<EW> oe(ends, old);
                if (oe.same(me)) {
                    if (atomicCAS(tab + 2 * p + 1, NONE, (uint32_t)e) != NONE || ((me.flags ^ oe.flags) & END_SIDE) == 0) {
                        atomicOr(err, DERR_BAD_GRAPH);
                    } else {
                        partner[e] = old;
                        partner[old] = (uint32_t)e;
                    }
                    break;
                }
                if (++p == base + t) p = base;
            }
        }
    }
}

// 2a: per entry x: its predecessor, its own bases w (label length - k) and whether it
// is a splitter (a head, a tail, or sampled); splitters get dense ids.  node[x] holds
// {pred, w} for an entry and {pred, sid | SPLIT} for a splitter (whose w goes to sw).
// Entry x = lm-tig x/2 entered through end x&1 (0: u, read forward; 1: v, reverse); its
// predecessor left its lm-tig through the end paired with x's entry end, and its
// successor entered through the end paired with x's exit end.
__global__ void __launch_bounds__(256) k_rs_init(const uint32_t* __restrict__ lens, uint64_t n,
                                                  const uint32_t* __restrict__ partner, uint32_t k, uint32_t sample_mask,
                                                  uint2* node, uint32_t* sx, uint32_t* sw, unsigned long long* n_split,
                                                  uint32_t* err) {
    __shared__ uint32_t wsum[8];
    __shared__ unsigned long long bbase;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t n2 = 2 * n, stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n2; base += stride) {   // block-uniform trips
        const uint64_t x = base + threadIdx.x;
        bool split = false;
        uint32_t pred = NONE, w = 0;
        if (x < n2) {
            const uint32_t q = partner[x];
            pred = q == NONE ? NONE : (q ^ 1u);
            const bool tail = partner[x ^ 1] == NONE;
            split = pred == NONE || tail || (mix64(x + 0x2545F4914F6CDD1Dull) & sample_mask) == 0;
            w = lens[x >> 1] - k;
            if (w & SPLIT) atomicOr(err, DERR_WALK_LIMIT);   // an lm-tig of 2^31 bases
        }
        // one atomic per block for the splitters' ids
        const uint32_t bal = __ballot_sync(0xffffffffu, split);
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t tot = 0;
            for (uint32_t v = 0; v < 8; ++v) { const uint32_t c = wsum[v]; wsum[v] = tot; tot += c; }
            bbase = tot ? atomicAdd(n_split, (unsigned long long)tot) : 0ull;
        }
        __syncthreads();
        if (x < n2) {
            if (split) {
                const uint32_t sid = (uint32_t)(bbase + wsum[wid] + __popc(bal & ((1u << lane) - 1)));
                sx[sid] = (uint32_t)x;
                sw[sid] = w;
                node[x] = make_uint2(pred, sid | SPLIT);
            } else {
                node[x] = make_uint2(pred, w);
            }
        }
        __syncthreads();
    }
}

// 2b: from every splitter, walk back through the entries before it to the previous
// splitter: each entry passed gets {splitter | OWNED, bases from its own start to the
// splitter's} in place of its node word (read just before, so the write hits L2), and
// the splitter links to the previous one (or is a head).  Warps take splitters from a
// counter, 32 at a time and in order, so the walks in flight stay near each other in
// memory; a lane takes the warp's next splitter as soon as its walk ends.
__global__ void __launch_bounds__(256) k_rs_walk(const uint32_t* __restrict__ sx, const uint32_t* __restrict__ sw,
                                                  const unsigned long long* __restrict__ n_split, uint2* node, RankRec* S,
                                                  unsigned long long* pool_ctr, uint64_t limit, uint32_t* err) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1;
    const uint64_t ns = *n_split;
    unsigned long long pool_next = 0, pool_end = 0;   // warp-uniform: splitters not yet taken
    bool exhausted = false;
    uint32_t cur = NONE, y = NONE;
    unsigned long long B = 0;
    for (uint64_t it = 0; it < limit; ++it) {
        uint32_t need = __ballot_sync(0xffffffffu, cur == NONE);
        while (need && !exhausted) {
            if (pool_next == pool_end) {
                unsigned long long b0 = 0;
                if (lane == 0) b0 = atomicAdd(pool_ctr, 32ull);
                b0 = __shfl_sync(0xffffffffu, b0, 0);
                if (b0 >= ns) { exhausted = true; break; }
                pool_next = b0;
                pool_end = b0 + 32 < ns ? b0 + 32 : ns;
            }
            const uint32_t avail = (uint32_t)(pool_end - pool_next);
            const uint32_t rank = __popc(need & lt);
            if (((need >> lane) & 1) && rank < avail) {
                cur = (uint32_t)(pool_next + rank);
                const uint32_t x = sx[cur];
                y = node[x].x;
                B = 0;
                if (y == NONE) { S[cur] = RankRec{NONE, x, 0ull}; cur = NONE; }   // a head
            }
            const uint32_t took = __popc(need) < avail ? __popc(need) : avail;
            pool_next += took;
            need = __ballot_sync(0xffffffffu, cur == NONE);
        }
        if (__all_sync(0xffffffffu, cur == NONE)) return;   // only when the counter is spent
        if (cur == NONE) continue;
        const uint2 ny = node[y];
        if (ny.y & SPLIT) {
            const uint32_t sid = ny.y & ~SPLIT;
            S[cur] = RankRec{sid, 0u, B + sw[sid]};
            cur = NONE;
            continue;
        }
        B += ny.y;
        if (B & SPLIT) { atomicOr(err, DERR_WALK_LIMIT); B = 0; }   // 2^31 bases between two splitters
        node[y] = make_uint2(cur | OWNED, (uint32_t)B);
        y = ny.x;
        if (y == NONE) {   // heads are splitters: unreachable on a valid graph
            atomicOr(err, DERR_BAD_GRAPH);
            S[cur] = RankRec{NONE, sx[cur], 0ull};
            cur = NONE;
        }
    }
    atomicOr(err, DERR_WALK_LIMIT);   // step bound exceeded
}

// One pointer-jumping round over the splitters (double-buffered); counts the entries
// still unresolved.
__global__ void k_ut_rank_round(const unsigned long long* __restrict__ n_split, const RankRec* __restrict__ X,
                                RankRec* X2, unsigned long long* active) {
    const uint64_t n2 = *n_split;
    uint32_t act = 0;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n2; x += (uint64_t)gridDim.x * blockDim.x) {
        RankRec r = X[x];
        if (r.P != NONE) {   // one 16-byte gather of the predecessor's record
            const RankRec q = X[r.P];
            r.P = q.P; r.R = q.R; r.A += q.A;
            act += q.P != NONE;
        }
        X2[x] = r;
    }
    if (!active) return;
    for (int d = 16; d; d >>= 1) act += __shfl_down_sync(0xffffffffu, act, d);
    if ((threadIdx.x & 31) == 0 && act) atomicAdd(active, (unsigned long long)act);
}

// 2c: every entry's rank from its splitter's: head entry and bases before it.  Entries
// on closed chains keep a predecessor (P != NONE); entries no walk passed are on closed
// chains without a splitter.
__global__ void k_rs_final(uint64_t n2, const uint2* __restrict__ node, RankRec* X, const RankRec* __restrict__ S) {
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n2; x += (uint64_t)gridDim.x * blockDim.x) {
        const uint2 nd = node[x];
        if (nd.y & SPLIT) {
            X[x] = S[nd.y & ~SPLIT];
        } else if (nd.x != NONE && (nd.x & OWNED)) {
            const RankRec q = S[nd.x & ~OWNED];
            X[x] = RankRec{q.P, q.R, q.A - nd.y};
        } else {
            X[x] = RankRec{UNOWNED, 0u, 0ull};
        }
    }
}

__device__ __forceinline__ char comp_char(char c) { return c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'A'; }
// base i of lm-tig x's label read in the direction of entry x
__device__ __forceinline__ char oriented(const char* lab, uint32_t len, uint32_t x, uint32_t i) {
    return (x & 1) ? comp_char(lab[len - 1 - i]) : lab[i];
}

// 3: per chain, once (by the lm-tig heading the list the host collator walks): flip the
// list when its reverse complement starts with a smaller k-mer (ties keep the walk).
__global__ void k_ut_flip(const uint32_t* __restrict__ lens, const char* const* __restrict__ label, uint64_t n,
                          const RankRec* __restrict__ X, uint32_t k, uint8_t* flipb) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t e0 = (uint32_t)(2 * i), e1 = e0 + 1;
        const RankRec x0 = X[e0], x1 = X[e1];
        if (x0.P != NONE || x1.P != NONE) continue;     // on a closed chain
        const uint32_t e = x0.R < x1.R ? e0 : e1;
        const uint32_t h = e == e0 ? x0.R : x1.R;
        if (h != e) continue;                           // not the head of its list
        const uint32_t t = (e == e0 ? x1.R : x0.R) ^ 1u;   // the entry of the list's tail
        const char* lh = label[h >> 1];
        const char* lt = label[t >> 1];
        const uint32_t nh = lens[h >> 1], nt = lens[t >> 1];
        bool flip = false;
        for (uint32_t j = 0; j < k; ++j) {
            const char a = oriented(lh, nh, h, j);
            const char b = comp_char(oriented(lt, nt, t, nt - 1 - j));
            if (a != b) { flip = b < a; break; }
        }
        flipb[i] = flip;
    }
}

// 4a: per lm-tig, the final entry; per final tail, the unitig's FASTA record.
// final[i] = chosen entry of lm-tig i, or NONE when i lies on a cycle.
__global__ void k_ut_choose(const uint32_t* __restrict__ lens, const char* const* __restrict__ label, uint64_t n,
                            const uint32_t* __restrict__ partner, const RankRec* __restrict__ X, uint32_t k,
                            uint32_t* fin, unsigned long long* out_off, unsigned long long* cursor, unsigned long long* n_units,
                            unsigned long long* n_cyc, const uint32_t* __restrict__ job,
                            const unsigned long long* __restrict__ job_out_base, unsigned long long* job_cur,
                            const uint8_t* __restrict__ flipb) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        bool tail = false;
        unsigned long long L = 0;
        uint32_t head = NONE, f = NONE;
        if (i < n) {
            const uint32_t e0 = (uint32_t)(2 * i), e1 = e0 + 1;
            const RankRec x0 = X[e0], x1 = X[e1];
            if (x0.P != NONE || x1.P != NONE) {   // on a closed chain
                fin[i] = NONE;
                atomicAdd(n_cyc, 1ull);
            } else {
                const uint32_t e = x0.R < x1.R ? e0 : e1;   // the list the host collator walks
                const bool flip = flipb[(e == e0 ? x0.R : x1.R) >> 1];   // decided by that list's head
                f = flip ? (e ^ 1u) : e;
                fin[i] = f;
                // the final list's tail: its exit end has no partner (or is phi)
                if (partner[f ^ 1u] == NONE) {
                    tail = true;
                    const RankRec xf = f == e0 ? x0 : x1;
                    head = xf.R;
                    L = xf.A + lens[f >> 1];   // bases before the tail + its whole label
                }
            }
        }
        const unsigned long long want = tail ? L + 4 : 0;
        if (!job) {   // warp-aggregated reservation of the unitigs' records
            unsigned long long x = want;
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= (uint32_t)d) x += y;
            }
            const unsigned long long tot = __shfl_sync(0xffffffffu, x, 31);
            unsigned long long b0 = 0;
            if (lane == 0 && tot) b0 = atomicAdd(cursor, tot);
            b0 = __shfl_sync(0xffffffffu, b0, 0);
            if (tail) {
                out_off[head] = b0 + x - want;
                atomicAdd(n_units, 1ull);
            }
        } else {      // per job: lanes of one job reserve together from its cursor
            const uint32_t jb = tail ? job[i] : NONE;
            unsigned long long pre = 0, tot = 0, cnt = 0;
            uint32_t leader = 32;
            for (uint32_t l = 0; l < 32; ++l) {
                const unsigned long long v = __shfl_sync(0xffffffffu, want, l);
                const uint32_t jl = __shfl_sync(0xffffffffu, jb, l);
                if (jl == jb) { tot += v; ++cnt; if (l < lane) pre += v; if (leader == 32) leader = l; }
            }
            unsigned long long b0 = 0;
            if (tail && leader == lane) {
                b0 = atomicAdd(job_cur + (size_t)jb * JOB_CUR_STRIDE, tot);
                atomicAdd(job_cur + (size_t)jb * JOB_CUR_STRIDE + 1, cnt);
            }
            b0 = __shfl_sync(0xffffffffu, b0, leader & 31);
            if (tail) {
                out_off[head] = job_out_base[jb] + b0 + pre;
                atomicAdd(n_units, 1ull);
            }
        }
    }
}

// 4b: every lm-tig's label at its place; heads write the header, tails the newline.
// An lm-tig writes only the bases its successor does not: all but its last k (the
// vertex they share, which the successor writes), or all of them at the tail.  Each
// thread resolves one lm-tig's source and destination and copies short pieces itself
// (eight loads in flight before the stores); the warp copies long ones together.
__global__ void k_ut_write(const uint32_t* __restrict__ lens, const char* const* __restrict__ label, uint64_t n,
                           const uint32_t* __restrict__ fin, const uint32_t* __restrict__ partner,
                           const RankRec* __restrict__ X, const unsigned long long* __restrict__ out_off, uint32_t k,
                           char* out) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {   // warp-uniform trips
        const uint64_t i = base + threadIdx.x;
        uint32_t f = NONE, len = 0, nc = 0;
        const char* lab = nullptr;
        char* dst = nullptr;
        if (i < n) {
            f = fin[i];
            if (f != NONE) {
                len = lens[i];
                lab = label[i];
                const RankRec xf = X[f];
                char* rec = out + out_off[xf.R];
                dst = rec + 3 + xf.A;
                if (xf.R == f) { rec[0] = '>'; rec[1] = '0'; rec[2] = '\n'; }
                const bool tail = partner[f ^ 1u] == NONE;
                nc = tail ? len : len - k;
                if (tail) dst[len] = '\n';
            }
        }
        const bool longer = nc > 64;
        if (!longer) {
            for (uint32_t j0 = 0; j0 < nc; j0 += 8) {
                char c[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) c[u] = j0 + u < nc ? oriented(lab, len, f, j0 + u) : 0;
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (j0 + u < nc) dst[j0 + u] = c[u];
            }
        }
        for (uint32_t todo = __ballot_sync(0xffffffffu, longer); todo; todo &= todo - 1) {
            const int l = __ffs(todo) - 1;
            const char* sl = (const char*)__shfl_sync(0xffffffffu, (unsigned long long)lab, l);
            char* dl = (char*)__shfl_sync(0xffffffffu, (unsigned long long)dst, l);
            const uint32_t ll = __shfl_sync(0xffffffffu, len, l), cl = __shfl_sync(0xffffffffu, nc, l);
            const uint32_t fl = __shfl_sync(0xffffffffu, f, l);
            for (uint32_t j0 = 0; j0 < cl; j0 += 128) {
                char c[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t j = j0 + 32 * u + lane;
                    c[u] = j < cl ? oriented(sl, ll, fl, j) : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t j = j0 + 32 * u + lane;
                    if (j < cl) dl[j] = c[u];
                }
            }
        }
    }
}

// ---- closed chains (cycles), joined on the device ----
// The lm-tigs left on closed chains (fin == NONE) are numbered 0..m-1; entry X = 2 c + d
// of cycle lm-tig c is it entered by its end d (0: u, read forward).  X's successor
// enters the lm-tig paired with X's exit end.  Every closed chain appears twice, once per
// orientation; the one whose smallest original entry id is even is kept.  Pointer
// jumping gives each kept entry its chain's head (that smallest entry) and its offset in
// the chain's circular text C (T bases: every lm-tig adds its label minus the k bases it
// shares with the next).  One CTA per chain then finds the smallest k-mer of C over both
// strands and writes C rotated to start there, in that strand, k-1 bases longer than T
// (canonicalize_cycle, include/Unitig_Collator.hpp:367-407): a chain's k-mers are all
// distinct vertices, so the smallest is unique and the result does not depend on where the
// walk started.
constexpr uint32_t CYC = 0x80000000u;

__global__ void k_cy_number(uint32_t* fin, uint64_t n, uint32_t* cyc_lm, unsigned long long* cnt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (fin[i] != NONE) continue;
        const uint32_t c = (uint32_t)atomicAdd(cnt, 1ull);
        fin[i] = CYC | c;
        cyc_lm[c] = (uint32_t)i;
    }
}

struct CyArgs {
    const uint32_t* len; const char* const* label; const uint32_t* partner; const uint32_t* fin;
    const uint32_t* cyc_lm; uint64_t m2;    // entries: 2 x cycle lm-tigs
    const uint32_t* job;                    // batch: each gathered lm-tig's job (nullptr: one job)
    uint32_t* rec_job;                      // per cycle record (in head order): its job
    uint32_t k;
    uint32_t *succ, *jmp0, *jmp1, *mn0, *mn1, *head;
    unsigned long long *w, *acc0, *acc1, *pos;
    uint32_t* err;
};

// successor, first jump, own original entry id, own bases
__global__ void k_cy_init(CyArgs a) {
    for (uint64_t X = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; X < a.m2; X += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = a.cyc_lm[X >> 1], d = (uint32_t)(X & 1);
        const uint32_t y = a.partner[2 * i + (d ^ 1u)];          // the entry after i's exit end
        uint32_t nx = (uint32_t)X;
        if (y == NONE || !(a.fin[y >> 1] & CYC) || a.fin[y >> 1] == NONE) atomicOr(a.err, DERR_BAD_GRAPH);
        else nx = 2 * (a.fin[y >> 1] & ~CYC) + (y & 1);
        a.succ[X] = nx; a.jmp0[X] = nx;
        a.mn0[X] = 2 * i + d;
        const uint32_t len = a.len[i];
        a.w[X] = len >= a.k ? len - a.k : 0;
    }
}

// one round of minimum propagation along the chain (double-buffered)
__global__ void k_cy_min(uint64_t m2, const uint32_t* __restrict__ jmp, const uint32_t* __restrict__ mn, uint32_t* jmp2,
                         uint32_t* mn2) {
    for (uint64_t X = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; X < m2; X += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = jmp[X];
        const uint32_t a = mn[X], b = mn[j];
        mn2[X] = a < b ? a : b;
        jmp2[X] = jmp[j];
    }
}

// head of every kept entry (NONE for the mirror orientation); the suffix-sum start
__global__ void k_cy_head(CyArgs a, const uint32_t* __restrict__ mn) {
    for (uint64_t X = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; X < a.m2; X += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t e = mn[X];
        uint32_t H = NONE;
        if (!(e & 1)) H = 2 * (a.fin[e >> 1] & ~CYC) + (e & 1);
        a.head[X] = H;
        const bool is_h = H == (uint32_t)X;
        a.jmp0[X] = is_h ? (uint32_t)X : a.succ[X];
        a.acc0[X] = (H == NONE || is_h) ? 0ull : a.w[X];
    }
}

// one round of suffix sums towards the head (the head is terminal: a self-loop of weight 0)
__global__ void k_cy_sum(uint64_t m2, const uint32_t* __restrict__ head, const uint32_t* __restrict__ jmp,
                         const unsigned long long* __restrict__ acc, uint32_t* jmp2, unsigned long long* acc2) {
    for (uint64_t X = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; X < m2; X += (uint64_t)gridDim.x * blockDim.x) {
        if (head[X] == NONE) continue;
        const uint32_t j = jmp[X];
        acc2[X] = acc[X] + acc[j];
        jmp2[X] = jmp[j];
    }
}

// every kept entry's offset in its chain's text; per head the chain's length T and its
// space in the scratch text and in the output (">0\n" + T + k - 1 bases + "\n")
__global__ void k_cy_place(CyArgs a, const unsigned long long* __restrict__ D, unsigned long long* T_of,
                           unsigned long long* scr_off, unsigned long long* out_off, uint32_t* heads,
                           unsigned long long* cur) {   // cur: [0] scratch bytes, [1] output bytes, [2] chains
    for (uint64_t X = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; X < a.m2; X += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t H = a.head[X];
        if (H == NONE) continue;
        const unsigned long long T = a.w[H] + D[a.succ[H]];
        a.pos[X] = X == H ? 0ull : T - D[X];
        if (X == H) {
            T_of[X] = T;
            scr_off[X] = atomicAdd(cur, T);
            out_off[X] = atomicAdd(cur + 1, T + a.k - 1 + 4);
            const unsigned long long hi = atomicAdd(cur + 2, 1ull);
            heads[hi] = (uint32_t)X;
            a.rec_job[hi] = a.job ? a.job[a.cyc_lm[X >> 1]] : 0u;
        }
    }
}

// every kept entry's label (in its orientation), all but its last k bases, into the text
__global__ void k_cy_text(CyArgs a, const unsigned long long* __restrict__ scr_off, char* scr) {
    for (uint64_t X = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; X < a.m2; X += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t H = a.head[X];
        if (H == NONE) continue;
        const uint32_t i = a.cyc_lm[X >> 1], len = a.len[i];
        const char* lab = a.label[i];
        char* dst = scr + scr_off[H] + a.pos[X];
        const uint64_t wx = a.w[X];
        for (uint64_t t = 0; t < wx; ++t) dst[t] = oriented(lab, len, (uint32_t)(X & 1), (uint32_t)t);
    }
}

__device__ __forceinline__ uint32_t code_of(char c) { return c == 'A' ? 0u : c == 'C' ? 1u : c == 'G' ? 2u : 3u; }
// (k-mer words from the highest, index, strand) ordered lexicographically: the k-mer
// first (big-endian 2-bit, so numeric order is character order), then where it was found.
// Four words hold any k <= 127.
struct CyKey { unsigned long long w[4]; unsigned long long i; uint32_t s; };
__device__ __forceinline__ bool cy_less(const CyKey& a, const CyKey& b) {
#pragma unroll
    for (int j = 3; j >= 0; --j)
        if (a.w[j] != b.w[j]) return a.w[j] < b.w[j];
    if (a.i != b.i) return a.i < b.i;
    return a.s < b.s;
}

// one CTA per chain: the smallest k-mer over both strands, then the rotated record
__global__ void __launch_bounds__(256) k_cy_rotate(const uint32_t* __restrict__ heads, const unsigned long long* __restrict__ n_heads,
                                                   const unsigned long long* __restrict__ T_of,
                                                   const unsigned long long* __restrict__ scr_off,
                                                   const unsigned long long* __restrict__ out_off, const char* scr,
                                                   uint32_t k, char* out) {
    __shared__ CyKey red[8];
    const uint64_t nh = *n_heads;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t kb = 2 * k;   // bits of a k-mer (k <= 127: at most 254)
    unsigned long long mask[4];   // the bits of each word a k-mer uses
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int left = (int)kb - 64 * j;
        mask[j] = left >= 64 ? ~0ull : left <= 0 ? 0ull : ((1ull << left) - 1);
    }
    const uint32_t top = (kb - 2) >> 6, top_sh = (kb - 2) & 63;   // where the rc's first base goes
    for (uint64_t h = blockIdx.x; h < nh; h += gridDim.x) {
        const uint32_t H = heads[h];
        const unsigned long long T = T_of[H];
        const char* C = scr + scr_off[H];
        // positions [j0, j1) of this thread; the k-mer at j covers C[j .. j+k) circularly
        const unsigned long long j0 = T * threadIdx.x / blockDim.x, j1 = T * (threadIdx.x + 1) / blockDim.x;
        CyKey best{{~0ull, ~0ull, ~0ull, ~0ull}, ~0ull, 1u};
        unsigned long long f[4] = {0, 0, 0, 0}, r[4] = {0, 0, 0, 0};   // forward / reverse-complement k-mer
        auto push = [&](uint32_t b) {   // appends base b to the forward k-mer, prepends comp(b) to the rc
#pragma unroll
            for (int j = 3; j > 0; --j) f[j] = ((f[j] << 2) | (f[j - 1] >> 62)) & mask[j];
            f[0] = ((f[0] << 2) | b) & mask[0];
            const unsigned long long cb = 3u - b;
#pragma unroll
            for (int j = 0; j < 3; ++j) r[j] = (r[j] >> 2) | (r[j + 1] << 62);
            r[3] >>= 2;
#pragma unroll
            for (int j = 0; j < 4; ++j) r[j] |= top == (uint32_t)j ? cb << top_sh : 0ull;
        };
        if (j0 < j1) {
            for (uint32_t t = 0; t + 1 < k; ++t) push(code_of(C[(j0 + t) % T]));
            for (unsigned long long j = j0; j < j1; ++j) {
                push(code_of(C[(j + k - 1) % T]));
                const CyKey fk{{f[0], f[1], f[2], f[3]}, j, 0u}, rk{{r[0], r[1], r[2], r[3]}, T - 1 - j, 1u};
                if (cy_less(fk, best)) best = fk;
                if (cy_less(rk, best)) best = rk;
            }
        }
        for (int d = 16; d; d >>= 1) {
            CyKey o;
#pragma unroll
            for (int j = 0; j < 4; ++j) o.w[j] = __shfl_down_sync(0xffffffffu, best.w[j], d);
            o.i = __shfl_down_sync(0xffffffffu, best.i, d); o.s = __shfl_down_sync(0xffffffffu, best.s, d);
            if (cy_less(o, best)) best = o;
        }
        if (lane == 0) red[wid] = best;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (uint32_t v = 1; v < blockDim.x / 32; ++v) if (cy_less(red[v], red[0])) red[0] = red[v];
        }
        __syncthreads();
        const CyKey b = red[0];
        char* o = out + out_off[H];
        const unsigned long long L = T + k - 1;
        if (threadIdx.x == 0) { o[0] = '>'; o[1] = '0'; o[2] = '\n'; o[3 + L] = '\n'; }
        // strand 0: C from b.i; strand 1: the reverse complement read so that its base u is
        // comp(C[(k - 2 - b.i - u) mod T])
        for (unsigned long long u = threadIdx.x; u < L; u += blockDim.x) {
            char c;
            if (b.s == 0) c = C[(b.i + u) % T];
            else {
                const long long q = ((long long)k - 2 - (long long)b.i - (long long)u) % (long long)T;
                c = comp_char(C[q < 0 ? q + (long long)T : q]);
            }
            o[3 + u] = c;
        }
        __syncthreads();
    }
}

}  // namespace

bool UnitigBuffers::ensure(uint64_t n) {
    // vertex table: 4 slots per lm-tig (at most half full: 2 ends per lm-tig); after
    // pairing it holds the splitters' second ranking buffer (up to 2n records)
    const uint64_t t = 4 * n + 64;
    const uint64_t n2 = 2 * n + 2;
    if (!b_label.ensure(8 * (n + 1)) || !b_tab.ensure(sizeof(EndSlot) * t) ||
        !b_partner.ensure(4 * n2) || !b_X0.ensure(sizeof(RankRec) * n2) || !b_X1.ensure(sizeof(RankRec) * n2) ||
        !b_fin.ensure(4 * (n + 1)) || !b_sx.ensure(4 * n2) || !b_sw.ensure(4 * n2) ||
        !b_off.ensure(8 * n2) || !b_words.ensure(64) || !b_job.ensure(4 * (n + 1)) || !b_flip.ensure(n + 1) ||
        !b_len.ensure(4 * (n + 1)) || !b_ends.ensure(16ull * end_words * (n + 1)))
        return false;
    len = b_len.as<uint32_t>();
    ends = b_ends.as<ulonglong2>();
    job = b_job.as<uint32_t>();
    flipb = b_flip.as<uint8_t>();
    label = (const char**)b_label.p; tab = b_tab.p; tab_n = t;
    partner = b_partner.as<uint32_t>(); X[0] = b_X0.p; X[1] = b_X1.p;
    fin = b_fin.as<uint32_t>(); out_off = b_off.as<unsigned long long>();
    sx = b_sx.as<uint32_t>();
    sw = b_sw.as<uint32_t>();
    words = b_words.as<unsigned long long>();
    return true;
}

int collate_cycles_on_device(UnitigBuffers& ub, uint64_t n, uint64_t m, uint32_t k, uint32_t* err, DevBuf& work,
                             DevBuf& scratch, DevBuf& out, cudaStream_t s, uint64_t& out_bytes, uint64_t& n_cycles,
                             const uint32_t* job, std::vector<CycleRecord>* records) {
    out_bytes = 0; n_cycles = 0;
    if (records) records->clear();
    if (m == 0) return CFG_OK;
    if (2 * m >= CYC) return CFG_ERR_BAD_INPUT;
    const uint64_t m2 = 2 * m;
    // per entry: succ, jmp0, jmp1, mn0, mn1, head (u32); w, acc0, acc1, pos, T, scratch and
    // output offsets (u64); heads (u32); the cycle lm-tigs (u32, m); three counters
    const size_t need = m2 * (8 * 4 + 7 * 8) + 4 * m + 512;   // + each array's 16-byte alignment
    if (!work.ensure(need)) return CFG_ERR_OOM;
    unsigned char* p = work.as<unsigned char>();
    auto take = [&](size_t bytes) { unsigned char* q = p; p += (bytes + 15) & ~(size_t)15; return q; };
    unsigned long long* cur = (unsigned long long*)take(32);
    CyArgs a{};
    a.len = ub.len; a.label = ub.label; a.partner = ub.partner; a.fin = ub.fin; a.m2 = m2; a.k = k; a.err = err;
    a.w = (unsigned long long*)take(8 * m2); a.acc0 = (unsigned long long*)take(8 * m2);
    a.acc1 = (unsigned long long*)take(8 * m2); a.pos = (unsigned long long*)take(8 * m2);
    unsigned long long* T_of = (unsigned long long*)take(8 * m2);
    unsigned long long* scr_off = (unsigned long long*)take(8 * m2);
    unsigned long long* out_off = (unsigned long long*)take(8 * m2);
    a.succ = (uint32_t*)take(4 * m2); a.jmp0 = (uint32_t*)take(4 * m2); a.jmp1 = (uint32_t*)take(4 * m2);
    a.mn0 = (uint32_t*)take(4 * m2); a.mn1 = (uint32_t*)take(4 * m2); a.head = (uint32_t*)take(4 * m2);
    uint32_t* heads = (uint32_t*)take(4 * m2);
    a.rec_job = (uint32_t*)take(4 * m2);
    uint32_t* cyc_lm = (uint32_t*)take(4 * m);
    a.cyc_lm = cyc_lm; a.job = job;
    if (cudaMemsetAsync(cur, 0, 32, s) != cudaSuccess) return CFG_ERR_CUDA;
    const unsigned grid = (unsigned)std::min<uint64_t>(148ull * 8, (m2 + 255) / 256 + 1);
    k_cy_number<<<148 * 4, 256, 0, s>>>(ub.fin, n, cyc_lm, cur + 3);   // cur: scratch, output, chains, lm-tigs
    k_cy_init<<<grid, 256, 0, s>>>(a);
    uint32_t rounds = 1;
    while ((1ull << rounds) < m2) ++rounds;
    ++rounds;
    uint32_t *jA = a.jmp0, *jB = a.jmp1, *mA = a.mn0, *mB = a.mn1;
    for (uint32_t r = 0; r < rounds; ++r) {
        k_cy_min<<<grid, 256, 0, s>>>(m2, jA, mA, jB, mB);
        std::swap(jA, jB); std::swap(mA, mB);
    }
    k_cy_head<<<grid, 256, 0, s>>>(a, mA);   // restarts jmp0 / acc0 for the sums
    jA = a.jmp0; jB = a.jmp1;
    unsigned long long *sA = a.acc0, *sB = a.acc1;
    for (uint32_t r = 0; r < rounds; ++r) {
        k_cy_sum<<<grid, 256, 0, s>>>(m2, a.head, jA, sA, jB, sB);
        std::swap(jA, jB); std::swap(sA, sB);
    }
    k_cy_place<<<grid, 256, 0, s>>>(a, sA, T_of, scr_off, out_off, heads, cur);
    unsigned long long h[3] = {0, 0, 0};
    if (cudaMemcpyAsync(h, cur, 24, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return CFG_ERR_CUDA;
    if (!scratch.ensure(h[0] + 16) || !out.ensure(h[1] + 16)) return CFG_ERR_OOM;
    k_cy_text<<<grid, 256, 0, s>>>(a, scr_off, scratch.as<char>());
    k_cy_rotate<<<(unsigned)std::min<unsigned long long>(std::max<unsigned long long>(h[2], 1), 148ull * 8), 256, 0, s>>>(
        heads, cur + 2, T_of, scr_off, out_off, scratch.as<char>(), k, out.as<char>());
    if (cudaGetLastError() != cudaSuccess) return CFG_ERR_CUDA;
    out_bytes = h[1]; n_cycles = h[2];
    if (records && h[2]) {   // where each record went and whose it is (head order)
        std::vector<uint32_t> hh(h[2]), hj(h[2]);
        std::vector<unsigned long long> off(m2), T(m2);
        if (cudaMemcpyAsync(hh.data(), heads, 4 * h[2], cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(hj.data(), a.rec_job, 4 * h[2], cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(off.data(), out_off, 8 * m2, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(T.data(), T_of, 8 * m2, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return CFG_ERR_CUDA;
        records->resize(h[2]);
        for (uint64_t i = 0; i < h[2]; ++i)
            (*records)[i] = CycleRecord{hj[i], off[hh[i]], T[hh[i]] + k - 1 + 4};
    }
    return CFG_OK;
}

int collate_device(const UnitigInput& in, UnitigBuffers& ub, cudaStream_t s, UnitigResult& res) {
    res = UnitigResult{};
    const uint64_t n = in.n;
    ub.end_words = in.k > 63 ? 4 : 2;
    if (!ub.ensure(n)) return CFG_ERR_OOM;
    if (cudaMemsetAsync(ub.words, 0, sizeof(unsigned long long) * 8, s) != cudaSuccess) return CFG_ERR_CUDA;
    // [0] output bytes, [1] unitigs, [2] cycle lm-tigs, [3] active entries, [4] splitters,
    // [5] insert tiles taken, [6] splitters taken by walks
    unsigned long long* cursor = ub.words;
    if (n == 0) return CFG_OK;
    if (2 * n >= SPLIT) return CFG_ERR_BAD_INPUT;   // entry ids are 31-bit
    const unsigned grid = 148 * 8;
    const uint32_t* job = in.jobs ? ub.job : nullptr;
    if (in.jobs)
        k_ut_gather_jobs<<<dim3(16, std::min<uint32_t>(in.n_jobs, 65535)), 256, 0, s>>>(
            in.job_lm, in.job_text, in.jobs, in.n_jobs, in.job_n, in.job_lm_base, ub.label, ub.job, ub.len, ub.ends, ub.end_words);
    else
        k_ut_gather<<<dim3(64, in.stripes), 256, 0, s>>>(in.lm, in.lm_slice, in.text, in.text_slice, in.lm_base, in.text_base,
                                                         in.stripe_cur, in.stripes, ub.label, ub.len, ub.ends, ub.end_words);
    if (cudaMemsetAsync(ub.tab, 0xff, sizeof(EndSlot) * ub.tab_n, s) != cudaSuccess ||
        cudaMemsetAsync(ub.partner, 0xff, 4 * 2 * n, s) != cudaSuccess)
        return CFG_ERR_CUDA;
    if (ub.end_words == 2)
        k_ut_insert<2><<<grid, 256, 0, s>>>(ub.ends, job, n, (uint32_t*)ub.tab, in.job_lm_base, in.job_n, cursor + 5,
                                            ub.partner, in.err);
    else
        k_ut_insert<4><<<grid, 256, 0, s>>>(ub.ends, job, n, (uint32_t*)ub.tab, in.job_lm_base, in.job_n, cursor + 5,
                                            ub.partner, in.err);
    // ranking: splitters, their walks, pointer jumping over the splitters, every entry
    RankRec* X = (RankRec*)ub.X[0];
    uint2* node = (uint2*)ub.out_off;                          // free until the records are reserved
    RankRec* Sb[2] = {(RankRec*)ub.X[1], (RankRec*)ub.tab};   // the vertex table is done with
    k_rs_init<<<grid, 256, 0, s>>>(ub.len, n, ub.partner, in.k, 15u, node, ub.sx, ub.sw, cursor + 4, in.err);
    k_rs_walk<<<grid, 256, 0, s>>>(ub.sx, ub.sw, cursor + 4, node, Sb[0], cursor + 6, 4 * n + 64, in.err);
    int cur = 0;
    unsigned long long last = ~0ull;
    for (int round = 0; round < 64; round += 2) {   // two rounds per look at the active count
        k_ut_rank_round<<<grid, 256, 0, s>>>(cursor + 4, Sb[cur], Sb[cur ^ 1], nullptr);
        cur ^= 1;
        if (cudaMemsetAsync(cursor + 3, 0, 8, s) != cudaSuccess) return CFG_ERR_CUDA;
        k_ut_rank_round<<<grid, 256, 0, s>>>(cursor + 4, Sb[cur], Sb[cur ^ 1], cursor + 3);
        cur ^= 1;
        res.rounds += 2;
        unsigned long long active = 0;
        if (cudaMemcpyAsync(&active, cursor + 3, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return CFG_ERR_CUDA;
        if (active == 0 || active == last) break;   // resolved, or only closed chains left
        last = active;
    }
    // an invalid graph stops here, before any record is reserved or written
    uint32_t e = 0;
    if (cudaMemcpyAsync(&e, in.err, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return CFG_ERR_CUDA;
    if (e & DERR_BAD_GRAPH) return CFG_ERR_STATE;
    if (e & DERR_WALK_LIMIT) return CFG_ERR_WALK_LIMIT;
    k_rs_final<<<grid, 256, 0, s>>>(2 * n, node, X, Sb[cur]);
    k_ut_flip<<<grid, 256, 0, s>>>(ub.len, ub.label, n, X, in.k, ub.flipb);
    k_ut_choose<<<grid, 256, 0, s>>>(ub.len, ub.label, n, ub.partner, X, in.k, ub.fin,
                                     ub.out_off, cursor, cursor + 1, cursor + 2, job, in.job_out_base, in.job_cur,
                                     ub.flipb);
    unsigned long long w[3] = {0, 0, 0};
    if (cudaMemcpyAsync(w, cursor, 24, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return CFG_ERR_CUDA;
    // a batch's output regions are sized by the caller before the call
    if (!in.jobs && !ub.ensure_out(w[0] + 16)) return CFG_ERR_OOM;
    k_ut_write<<<grid, 256, 0, s>>>(ub.len, ub.label, n, ub.fin, ub.partner, X, ub.out_off, in.k, ub.out);
    if (cudaGetLastError() != cudaSuccess) return CFG_ERR_CUDA;
    res.bytes = w[0]; res.n_units = w[1]; res.n_cycle_lmtigs = w[2];
    return CFG_OK;
}

}  // namespace cfg
