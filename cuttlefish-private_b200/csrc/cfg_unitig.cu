// cfg_unitig.cu -- lm-tigs joined into maximal unitigs on the device.
//
// The discontinuity-graph phases of dBG_Contractor::construct
// (Discontinuity_Graph_Contractor::contract, Contracted_Graph_Expander::expand,
// Unitig_Collator::collate; src/dBG_Contractor.cpp:73-101) for an in-memory edge
// set, as data-parallel steps over the lm-tigs of one run:
//   1. pair the lm-tig ends that meet at a discontinuity vertex (a hash table on the
//      vertex k-mer; a vertex carries at most one lm-tig on each side);
//   2. list ranking by pointer jumping over the 2n (lm-tig, direction) entries: each
//      entry's predecessor is the entry that leaves through its partner end; after
//      ~log2(chain length) rounds every entry knows its chain's head and the label
//      bases before it (each lm-tig adds its length minus the k-base overlap);
//   3. of the two mirror lists of a chain, take the one whose head end has the
//      smaller id (the host collator's walk), then flip it if its reverse complement
//      starts with a smaller k-mer (Maximal_Unitig::canonicalize,
//      include/Unitig_Collator.hpp:308-347);
//   4. reserve each unitig's FASTA record, and let every lm-tig copy its label (read
//      forward or reverse-complemented) to its offset -- neighbours write the shared
//      k-mer twice, with the same bytes.
// Entries that never reach a head lie on closed chains (cycles); those lm-tigs are
// handed back to the host collator, whose rotation rule they need (rare).
#include "cuttlefish_gpu.h"
#include "cfg_host.h"
#include "cfg_internal.h"

#include <algorithm>

namespace cfg {

namespace {

constexpr uint32_t NONE = 0xffffffffu;

struct EndSlot {   // hash slot of one vertex: its k-mer and the (at most two) lm-tig ends there
    unsigned long long k0, k1;
    uint32_t e0, e1;
    uint32_t ready, pad;
};

// One (lm-tig, direction) entry of the ranking: predecessor still to jump over (NONE
// once resolved), the farthest known ancestor (the head once resolved), and the label
// bases of the entries between them.
struct RankRec { uint32_t P, R; unsigned long long A; };

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z ^= z >> 33; z *= 0xFF51AFD7ED558CCDull;
    z ^= z >> 33; z *= 0xC4CEB9FE1A85EC53ull;
    z ^= z >> 33;
    return z;
}

__global__ void k_ut_tab_init(EndSlot* tab, uint64_t n) {
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
        tab[p].e0 = NONE; tab[p].e1 = NONE; tab[p].ready = 0;
    }
}

__device__ __forceinline__ bool is_phi(const LmtigOut& m, uint32_t end) { return (m.flags >> (end ? 3 : 2)) & 1; }
__device__ __forceinline__ uint32_t side_of(const LmtigOut& m, uint32_t end) { return (m.flags >> end) & 1; }

// 0: gather the striped lm-tigs into one array with their label addresses.
__global__ void k_ut_gather(const LmtigOut* lm, uint64_t lm_slice, const char* text, uint64_t text_slice,
                            const unsigned long long* __restrict__ lm_base, const unsigned long long* __restrict__ text_base,
                            const unsigned long long* __restrict__ stripe_cur, uint32_t stripes, LmtigOut* out,
                            const char** label) {
    for (uint32_t st = blockIdx.y; st < stripes; st += gridDim.y) {
        const unsigned long long n = stripe_cur[st * JOB_CUR_STRIDE + 2];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
            const LmtigOut m = lm[st * lm_slice + i];
            const uint64_t g = lm_base[st] + i;
            out[g] = m;
            label[g] = text + st * text_slice + (m.label_off - text_base[st]);
        }
    }
}

// 0 (batch): gather every job's lm-tigs from its regions; the job rides along.
__global__ void k_ut_gather_jobs(const LmtigOut* lm, const char* text, const JobOut* __restrict__ jobs, uint32_t n_jobs,
                                 const unsigned long long* __restrict__ job_n, const unsigned long long* __restrict__ job_lm_base,
                                 LmtigOut* out, const char** label, uint32_t* out_job) {
    for (uint32_t j = blockIdx.y; j < n_jobs; j += gridDim.y) {
        const unsigned long long n = job_n[j];
        const JobOut& J = jobs[j];
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
            const LmtigOut m = lm[J.lm_off + i];
            const uint64_t g = job_lm_base[j] + i;
            out[g] = m;
            label[g] = text + J.lm_text_off + m.label_off;
            out_job[g] = j;
        }
    }
}

// 1: every non-phi end into the vertex table; the second end at a vertex pairs.
// In a batch the vertex is (job, k-mer).
__global__ void k_ut_insert(const LmtigOut* __restrict__ lm, const uint32_t* __restrict__ job, uint64_t n, EndSlot* tab,
                            uint64_t mask, uint32_t* err) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < 2 * n; e += (uint64_t)gridDim.x * blockDim.x) {
        const LmtigOut& m = lm[e >> 1];
        const uint32_t end = (uint32_t)(e & 1);
        if (is_phi(m, end)) continue;
        const unsigned long long k0 = end ? m.v[0] : m.u[0], k1 = end ? m.v[1] : m.u[1];
        const uint32_t jb = job ? job[e >> 1] : 0u;
        uint64_t p = mix64(k0 ^ mix64(k1 + 0x9E3779B97F4A7C15ull) ^ mix64(jb + 0x632BE59BD9B4E019ull)) & mask;
        for (uint64_t probe = 0; probe <= mask; ++probe, p = (p + 1) & mask) {
            EndSlot& s = tab[p];
            const uint32_t old = atomicCAS(&s.e0, NONE, (uint32_t)e);
            if (old == NONE) {
                s.k0 = k0; s.k1 = k1; s.pad = jb;
                __threadfence();
                atomicExch(&s.ready, 1u);
                break;
            }
            uint32_t spin = 0;
            while (atomicAdd(&s.ready, 0u) == 0) {
                if (++spin > (1u << 22)) { atomicOr(err, DERR_CAS_LIMIT); return; }
            }
            __threadfence();
            if (*(volatile unsigned long long*)&s.k0 == k0 && *(volatile unsigned long long*)&s.k1 == k1 &&
                *(volatile uint32_t*)&s.pad == jb) {
                if (atomicCAS(&s.e1, NONE, (uint32_t)e) != NONE) atomicOr(err, DERR_BAD_GRAPH);   // a third end
                break;
            }
        }
    }
}

// 2: partners, and the first round of the ranking: each entry's predecessor entry.
// Entry x = lm-tig x/2 entered through end x&1 (0: u, read forward; 1: v, reverse).
__global__ void k_ut_pair(const LmtigOut* __restrict__ lm, const EndSlot* __restrict__ tab, uint64_t tab_n,
                          uint32_t* partner, uint32_t* err) {
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < tab_n; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = tab[p].e0, b = tab[p].e1;
        if (a == NONE || b == NONE) continue;
        if (side_of(lm[a >> 1], a & 1) == side_of(lm[b >> 1], b & 1)) { atomicOr(err, DERR_BAD_GRAPH); continue; }
        partner[a] = b; partner[b] = a;
    }
}

__global__ void k_ut_rank_init(const LmtigOut* __restrict__ lm, uint64_t n, const uint32_t* __restrict__ partner, uint32_t k,
                               RankRec* X) {
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < 2 * n; x += (uint64_t)gridDim.x * blockDim.x) {
        // the predecessor left its lm-tig through the end paired with x's entry end
        const uint32_t q = partner[x];
        const uint32_t pred = q == NONE ? NONE : (q ^ 1u);
        RankRec r;
        r.P = pred;
        r.R = pred == NONE ? (uint32_t)x : pred;
        r.A = pred == NONE ? 0ull : (unsigned long long)(lm[pred >> 1].label_len - k);
        X[x] = r;
    }
}

// One pointer-jumping round (double-buffered); counts the entries still unresolved.
__global__ void k_ut_rank_round(uint64_t n2, const RankRec* __restrict__ X, RankRec* X2, unsigned long long* active) {
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

__device__ __forceinline__ char comp_char(char c) { return c == 'A' ? 'T' : c == 'C' ? 'G' : c == 'G' ? 'C' : 'A'; }
// base i of lm-tig x's label read in the direction of entry x
__device__ __forceinline__ char oriented(const char* lab, uint32_t len, uint32_t x, uint32_t i) {
    return (x & 1) ? comp_char(lab[len - 1 - i]) : lab[i];
}

// 3: per chain, once (by the lm-tig heading the list the host collator walks): flip the
// list when its reverse complement starts with a smaller k-mer (ties keep the walk).
__global__ void k_ut_flip(const LmtigOut* __restrict__ lm, const char* const* __restrict__ label, uint64_t n,
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
        const uint32_t nh = lm[h >> 1].label_len, nt = lm[t >> 1].label_len;
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
__global__ void k_ut_choose(const LmtigOut* __restrict__ lm, const char* const* __restrict__ label, uint64_t n,
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
                    L = xf.A + lm[f >> 1].label_len;   // bases before the tail + its whole label
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
__global__ void k_ut_write(const LmtigOut* __restrict__ lm, const char* const* __restrict__ label, uint64_t n,
                           const uint32_t* __restrict__ fin, const uint32_t* __restrict__ partner,
                           const RankRec* __restrict__ X, const unsigned long long* __restrict__ out_off, char* out) {
    // one warp per lm-tig: lanes copy the label's bytes
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
        const uint32_t f = fin[i];
        if (f == NONE) continue;
        const uint32_t len = lm[i].label_len;
        const char* lab = label[i];
        const RankRec xf = X[f];
        char* rec = out + out_off[xf.R];
        char* dst = rec + 3 + xf.A;
        for (uint32_t j = lane; j < len; j += 32) dst[j] = oriented(lab, len, f, j);
        if (lane == 0) {
            if (xf.R == f) { rec[0] = '>'; rec[1] = '0'; rec[2] = '\n'; }
            if (partner[f ^ 1u] == NONE) dst[len] = '\n';
        }
    }
}

// Lm-tigs on closed chains, with their labels, into small arrays for the host collator.
__global__ void k_ut_cycles(const LmtigOut* __restrict__ lm, const char* const* __restrict__ label, uint64_t n,
                            const uint32_t* __restrict__ fin, LmtigOut* out, char* text, unsigned long long* cnt,
                            const uint32_t* __restrict__ job, uint32_t* out_job) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        if (fin[i] != NONE) continue;
        LmtigOut m = lm[i];
        const unsigned long long slot = atomicAdd(cnt, 1ull);
        const unsigned long long off = atomicAdd(cnt + 1, (unsigned long long)m.label_len);
        if (!text) continue;   // sizing pass
        for (uint32_t j = 0; j < m.label_len; ++j) text[off + j] = label[i][j];
        m.label_off = off;
        out[slot] = m;
        if (out_job) out_job[slot] = job ? job[i] : 0u;
    }
}

}  // namespace

bool UnitigBuffers::ensure(uint64_t n) {
    uint64_t t = 64;
    while (t < 4 * n) t <<= 1;   // vertex table at most half full (2n ends)
    const uint64_t n2 = 2 * n + 2;
    if (!b_lm.ensure(sizeof(LmtigOut) * (n + 1)) || !b_label.ensure(8 * (n + 1)) || !b_tab.ensure(sizeof(EndSlot) * t) ||
        !b_partner.ensure(4 * n2) || !b_X0.ensure(sizeof(RankRec) * n2) || !b_X1.ensure(sizeof(RankRec) * n2) ||
        !b_fin.ensure(4 * (n + 1)) ||
        !b_off.ensure(8 * n2) || !b_words.ensure(64) || !b_job.ensure(4 * (n + 1)) || !b_flip.ensure(n + 1))
        return false;
    job = b_job.as<uint32_t>();
    flipb = b_flip.as<uint8_t>();
    lm = b_lm.as<LmtigOut>(); label = (const char**)b_label.p; tab = b_tab.p; tab_n = t;
    partner = b_partner.as<uint32_t>(); X[0] = b_X0.p; X[1] = b_X1.p;
    fin = b_fin.as<uint32_t>(); out_off = b_off.as<unsigned long long>();
    words = b_words.as<unsigned long long>();
    return true;
}

int collate_cycles_device(const UnitigBuffers& ub, uint64_t n, LmtigOut* out, char* text, unsigned long long* cnt,
                          cudaStream_t s, uint32_t* out_job) {
    k_ut_cycles<<<148 * 4, 256, 0, s>>>(ub.lm, ub.label, n, ub.fin, out, text, cnt, ub.job, out_job);
    return cudaGetLastError() == cudaSuccess ? CFG_OK : CFG_ERR_CUDA;
}

int collate_device(const UnitigInput& in, UnitigBuffers& ub, cudaStream_t s, UnitigResult& res) {
    res = UnitigResult{};
    const uint64_t n = in.n;
    if (!ub.ensure(n)) return CFG_ERR_OOM;
    if (cudaMemsetAsync(ub.words, 0, sizeof(unsigned long long) * 4, s) != cudaSuccess) return CFG_ERR_CUDA;
    unsigned long long* cursor = ub.words;      // [0] output bytes, [1] unitigs, [2] cycle lm-tigs, [3] active
    if (n == 0) return CFG_OK;
    const unsigned grid = 148 * 8;
    EndSlot* tab = (EndSlot*)ub.tab;
    const uint32_t* job = in.jobs ? ub.job : nullptr;
    if (in.jobs)
        k_ut_gather_jobs<<<dim3(16, std::min<uint32_t>(in.n_jobs, 65535)), 256, 0, s>>>(
            in.job_lm, in.job_text, in.jobs, in.n_jobs, in.job_n, in.job_lm_base, ub.lm, ub.label, ub.job);
    else
        k_ut_gather<<<dim3(64, in.stripes), 256, 0, s>>>(in.lm, in.lm_slice, in.text, in.text_slice, in.lm_base, in.text_base,
                                                         in.stripe_cur, in.stripes, ub.lm, ub.label);
    k_ut_tab_init<<<grid, 256, 0, s>>>(tab, ub.tab_n);
    if (cudaMemsetAsync(ub.partner, 0xff, 4 * 2 * n, s) != cudaSuccess) return CFG_ERR_CUDA;
    k_ut_insert<<<grid, 256, 0, s>>>(ub.lm, job, n, tab, ub.tab_n - 1, in.err);
    k_ut_pair<<<grid, 256, 0, s>>>(ub.lm, tab, ub.tab_n, ub.partner, in.err);
    RankRec* Xb[2] = {(RankRec*)ub.X[0], (RankRec*)ub.X[1]};
    k_ut_rank_init<<<grid, 256, 0, s>>>(ub.lm, n, ub.partner, in.k, Xb[0]);
    int cur = 0;
    unsigned long long last = ~0ull;
    for (int round = 0; round < 64; round += 2) {   // two rounds per look at the active count
        k_ut_rank_round<<<grid, 256, 0, s>>>(2 * n, Xb[cur], Xb[cur ^ 1], nullptr);
        cur ^= 1;
        if (cudaMemsetAsync(cursor + 3, 0, 8, s) != cudaSuccess) return CFG_ERR_CUDA;
        k_ut_rank_round<<<grid, 256, 0, s>>>(2 * n, Xb[cur], Xb[cur ^ 1], cursor + 3);
        cur ^= 1;
        res.rounds += 2;
        unsigned long long active = 0;
        if (cudaMemcpyAsync(&active, cursor + 3, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return CFG_ERR_CUDA;
        if (active == 0 || active == last) break;   // resolved, or only closed chains left
        last = active;
    }
    k_ut_flip<<<grid, 256, 0, s>>>(ub.lm, ub.label, n, Xb[cur], in.k, ub.flipb);
    k_ut_choose<<<grid, 256, 0, s>>>(ub.lm, ub.label, n, ub.partner, Xb[cur], in.k, ub.fin,
                                     ub.out_off, cursor, cursor + 1, cursor + 2, job, in.job_out_base, in.job_cur,
                                     ub.flipb);
    unsigned long long w[3] = {0, 0, 0};
    if (cudaMemcpyAsync(w, cursor, 24, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return CFG_ERR_CUDA;
    // a batch's output regions are sized by the caller before the call
    if (!in.jobs && !ub.ensure_out(w[0] + 16)) return CFG_ERR_OOM;
    k_ut_write<<<grid, 256, 0, s>>>(ub.lm, ub.label, n, ub.fin, ub.partner, Xb[cur], ub.out_off, ub.out);
    if (cudaGetLastError() != cudaSuccess) return CFG_ERR_CUDA;
    res.bytes = w[0]; res.n_units = w[1]; res.n_cycle_lmtigs = w[2];
    return CFG_OK;
}

}  // namespace cfg
