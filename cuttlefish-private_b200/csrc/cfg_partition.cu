// cfg_partition.cu -- K1: weak super k-mer partitioning and bucket scatter.
//
// Restates Graph_Partitioner::process_chunk (src/Graph_Partitioner.cpp:505-597)
// with Min_Iterator<k-1> (include/Minimizer_Iterator.hpp:306-378) as a
// data-parallel sweep.  For every (k-1)-mer j of a fragment the subgraph is
// g_j = (min over its k-l l-mers of min(wyhash(l-mer), wyhash(rc(l-mer)))) & (G-1).
// The sequential cut rule (cut where g changes, or where the super (k-1)-mer
// reaches 2(k-1)-l bases) is equivalent to: pieces start at every g change and
// then every k-l (k-1)-mers inside a run of equal g.  So a run's pieces depend
// only on where the run starts, and a warp can own every run that starts in its
// stream segment, continuing past the segment's end until that run ends.
#include "cfg_device.cuh"
#include "cfg_internal.h"

#include <algorithm>

namespace cfg {

namespace {

constexpr int WARPS_PER_BLOCK = 8;
constexpr uint32_t STAGE = 256;       // records a warp gathers in shared memory per reservation
constexpr uint32_t MODW = 160;        // residues kept: the cut test indexes up to w - 1 + 32

__device__ __forceinline__ uint32_t lanemask_lt() { uint32_t m; asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m)); return m; }

__device__ __forceinline__ uint64_t lmer_at(const uint64_t* __restrict__ s, uint64_t p, uint32_t l) {
    return window64(s, p) >> (64 - 2 * l);
}

// min(hash(l-mer at p), hash(its reverse complement)).  With the reverse-complemented
// words at hand, the reverse complement is a second window: its first base is the
// l-mer's last, e = p + l - 1, at index 31 - (e mod 32) of rcw[e / 32], and it continues
// into rcw[e / 32 - 1] -- two loads and a funnel shift instead of a bit reversal per
// l-mer (this kernel is bound by the integer ALU pipe, not by loads).
__device__ __forceinline__ uint64_t lmer_hash_at(const PartitionArgs& a, uint64_t p, uint32_t l) {
    const uint64_t fw = lmer_at(a.packed, p, l);
    if (!a.rcw) return lmer_hash(fw, l, a.seed0);
    const uint64_t e = p + l - 1, w2 = e >> 5;
    const uint32_t j = 31 - (uint32_t)(e & 31);
    const uint64_t hi = __ldg(a.rcw + w2);
    const uint64_t win = j == 0 ? hi : (hi << (2 * j)) | (w2 ? __ldg(a.rcw + w2 - 1) >> (64 - 2 * j) : 0ull);
    const uint64_t rc = win >> (64 - 2 * l);
    const uint64_t x = wyhash8(fw, a.seed0), y = wyhash8(rc, a.seed0);
    return x < y ? x : y;
}

__global__ void k_rc_words(const uint64_t* __restrict__ packed, uint64_t w0, uint64_t w1, uint64_t* rcw) {
    for (uint64_t w = w0 + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < w1; w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t r = __brevll(packed[w]);                                             // bits reversed
        r = ((r >> 1) & 0x5555555555555555ull) | ((r & 0x5555555555555555ull) << 1);  // each base's two bits restored
        rcw[w] = ~r;                                                                  // complemented: b -> 3 - b
    }
}

// A warp's records wait in shared memory and are reserved in the flat array together:
// one atomic on the run's record cursor per STAGE records instead of one per 32 positions.
struct Stage { uint64_t* buf; uint32_t n; };
__device__ __forceinline__ void stage_flush(const PartitionArgs& a, Stage& st) {
    if (st.n == 0) return;
    const uint32_t lane = threadIdx.x & 31;
    unsigned long long b0 = 0;
    if (lane == 0) b0 = atomicAdd(a.rec_cursor, (unsigned long long)st.n);
    b0 = __shfl_sync(0xffffffffu, b0, 0);
    __syncwarp();
    for (uint32_t i = lane; i < st.n; i += 32) {
        const unsigned long long idx = b0 + i;
        if (idx < a.rec_cap) a.recs[idx] = st.buf[i]; else atomicOr(a.err, DERR_REC_OVERFLOW);
    }
    __syncwarp();
    st.n = 0;
}

// The value lane (lane - d) holds in this chunk, or for lanes < d the value lane
// (lane - d + 32) held in the previous chunk (0 <= d <= 31): each source lane supplies
// exactly one of the two, so one shuffle serves both.
__device__ __forceinline__ uint64_t from_back(uint64_t cur, uint64_t prev, uint32_t d, uint32_t lane) {
    return __shfl_sync(0xffffffffu, lane >= 32 - d ? prev : cur, (lane - d) & 31);
}
__device__ __forceinline__ uint64_t min64(uint64_t a, uint64_t b) { return a < b ? a : b; }

// The sparse table's depth E = floor(log2 w) is a template argument: levels 2^0 .. 2^E,
// none more (w = k - l <= 126: E <= 6).

// Processes the (k-1)-mer positions [j0, j1) of one fragment: emits every weak
// super k-mer whose run starts there.
// mod_w[x] = x % w for x < MODW (w <= 126): the cap-cut test without a division.
// hist: this fragment's job's histogram (the run's, or its job's slice of a batch's);
// nullptr when the bucket sort counts the records itself.
//
// Window minima with warp shuffles: in the chunk of (k-1)-mers base .. base+31, lane L
// holds the newest l-mer hash, at q = base + w - 1 + L.  Level i of a sparse table holds
// at position q - 2^i + 1 the minimum of the 2^i hashes starting there: the minimum of
// the lane's own level i-1 value and that of the lane 2^(i-1) before it (for the first
// lanes, from the previous chunk).  The window of (k-1)-mer j = q - w + 1 is then two
// overlapping blocks of 2^E hashes, E = floor(log2 w): min(level_E[j], level_E[q-2^E+1]),
// the second the lane's own value, the first that of the lane w - 2^E before it.
// O(log w) work per position, no shared memory.  For w >= 96 (E = 6, dq = w - 64 > 32)
// the second block starts two chunks back: level E of the chunk before the previous is kept.
template <int E>
__device__ void sweep_fragment(const PartitionArgs& a, const uint8_t* mod_w, uint64_t F0, uint32_t FL,
                               uint32_t j0, uint32_t j1, unsigned long long* hist, Stage& st) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t k = a.k, l = a.l, w = a.w;
    const uint32_t M = FL - k + 2;                 // (k-1)-mers in the fragment
    const uint32_t n_lmers = FL - l + 1;
    const uint32_t start = j0 == 0 ? 0 : j0 - 1;   // position j0-1 only primes the change test
    const uint32_t dq = w - (1u << E);
    // hash of l-mer q, or "none" (all ones, above every hash) outside the fragment
    auto hash_at = [&](int64_t q) -> uint64_t {   // a negative q wraps above every l-mer count: one compare
        return (uint64_t)q < (uint64_t)n_lmers ? lmer_hash_at(a, F0 + (uint64_t)q, l) : ~0ull;
    };
    uint64_t lv[E + 1], pv[E + 1];   // this chunk's / the previous chunk's level values
    uint64_t ppE = ~0ull;            // level E two chunks back (E = 6 only)
#pragma unroll
    for (int i = 0; i <= E; ++i) pv[i] = ~0ull;
    auto levels = [&](uint64_t h) -> uint64_t {   // adds this chunk's hashes; the window minimum
        lv[0] = h;
#pragma unroll
        for (int i = 1; i <= E; ++i) lv[i] = min64(lv[i - 1], from_back(lv[i - 1], pv[i - 1], 1u << (i - 1), lane));
        uint64_t m;
        if constexpr (E >= 6) {   // dq <= 63: the block's start lies in one of the two chunks before
            m = dq <= 32 ? min64(lv[E], from_back(lv[E], pv[E], dq, lane))
                         : min64(lv[E], from_back(pv[E], ppE, dq - 32, lane));
            ppE = pv[E];
        } else {
            m = min64(lv[E], from_back(lv[E], pv[E], dq, lane));
        }
#pragma unroll
        for (int i = 0; i <= E; ++i) pv[i] = lv[i];
        return m;
    };
    // prime the levels with the chunks before the first: their hashes reach back to l-mer
    // `start`, ceil((w - 1) / 32) chunks (at least one)
    for (int c = (int)max(1u, (w - 1 + 31) / 32); c >= 1; --c) levels(hash_at((int64_t)start - 32 * c + w - 1 + lane));

    bool active = false;
    uint32_t r0 = 0, last_cut = 0, last_cut_g = 0, last_cut_chg = 0, carry_g = 0;
    uint32_t carry_rem = 0;   // (base - start of the run in progress) % w

    // each chunk's new l-mer hash is computed one chunk ahead, so its loads and
    // multiplies overlap the window minima of the chunk before
    uint64_t h_next = hash_at((int64_t)start + w - 1 + lane);
    for (uint32_t base = start;; base += 32) {
        const uint64_t h = h_next;
        h_next = hash_at((int64_t)base + 32 + w - 1 + lane);
        const uint64_t m = levels(h);
        const uint32_t j = base + lane;
        const bool valid = j < M;
        const uint32_t g = valid ? (uint32_t)m & a.gmask : 0u;
        uint32_t gprev = __shfl_up_sync(0xffffffffu, g, 1);
        if (lane == 0) gprev = carry_g;
        const bool is_chg = valid && j >= j0 && (j == 0 || gprev != g);
        const uint32_t chg = __ballot_sync(0xffffffffu, is_chg);

        bool just_activated = false;
        uint32_t r0_lane = 0;
        if (!active) {
            if (chg == 0) {
                if (base + 32 >= j1 || base + 32 >= M) return;   // no run starts in [j0, j1)
                carry_g = __shfl_sync(0xffffffffu, g, 31);
                continue;
            }
            r0_lane = __ffs(chg) - 1;
            r0 = base + r0_lane;
            if (r0 >= j1) return;
            active = true; just_activated = true;
            last_cut = r0;
            last_cut_g = __shfl_sync(0xffffffffu, g, r0_lane);
            last_cut_chg = 1;
        }
        const uint32_t act_mask = just_activated ? (0xffffffffu << r0_lane) : 0xffffffffu;

        // run start of each position: highest change at or below it, else the carried one
        const uint32_t le = chg & (lanemask_lt() | (1u << lane));
        const uint32_t rem = le ? mod_w[lane - (31 - __clz(le))] : mod_w[carry_rem + lane];
        const bool is_cut = valid && ((act_mask >> lane) & 1) && (is_chg || rem == 0);
        uint32_t cut = __ballot_sync(0xffffffffu, is_cut);

        // stop at the first change at or past j1: the run it starts belongs to the next segment
        bool stopping = false;
        {
            const uint32_t past = __ballot_sync(0xffffffffu, valid && j >= j1);
            const uint32_t stop = chg & past;
            if (stop) {
                const uint32_t sl = __ffs(stop) - 1;
                cut &= (sl == 31) ? 0xffffffffu : ((2u << sl) - 1);
                stopping = true;
            }
        }
        uint32_t emit = cut;
        if (just_activated) emit &= ~(1u << r0_lane);

        // piece [c, c') ends at every emitting lane c' = j
        const uint32_t below = cut & lanemask_lt();
        const uint32_t pl = below ? (31 - __clz(below)) : 0;
        const uint32_t pg = __shfl_sync(0xffffffffu, g, pl);
        const uint32_t pchg = __shfl_sync(0xffffffffu, (uint32_t)is_chg, pl);
        const bool fin = !stopping && (base + 32 >= M);      // the fragment's last (k-1)-mer is in this chunk
        const uint32_t n_emit = __popc(emit) + (fin ? 1 : 0);
        if (st.n + n_emit > STAGE) stage_flush(a, st);
        const uint32_t slot0 = st.n;
        st.n += n_emit;
        if ((emit >> lane) & 1) {
            const uint32_t c = below ? base + pl : last_cut;
            const uint32_t cg = below ? pg : last_cut_g;
            const uint32_t cchg = below ? pchg : last_cut_chg;
            const uint32_t lj = c > 0;
            const uint32_t len = lj + (j - c + k - 2) + 1;
            const uint64_t r = rec_pack((uint32_t)(F0 + c - lj), len, lj & cchg, is_chg ? 1u : 0u, cg);
            st.buf[slot0 + __popc(emit & lanemask_lt())] = r;
            if (hist) atomicAdd(hist + cg, 1ull | ((unsigned long long)(len - k + 1) << 32));
        }
        // carries: last cut / run start of this chunk
        if (cut) {
            const uint32_t hl = 31 - __clz(cut);
            last_cut = base + hl;
            last_cut_g = __shfl_sync(0xffffffffu, g, hl);
            last_cut_chg = __shfl_sync(0xffffffffu, (uint32_t)is_chg, hl);
        }
        carry_rem = chg ? mod_w[32 - (31 - __clz(chg))] : mod_w[carry_rem + 32];
        carry_g = __shfl_sync(0xffffffffu, g, 31);
        if (fin && lane == 0) {   // final piece [last_cut, M): not joined on the right
            const uint32_t c = last_cut, lj = c > 0;
            const uint32_t len = lj + (FL - c);
            const uint64_t r = rec_pack((uint32_t)(F0 + c - lj), len, lj & last_cut_chg, 0, last_cut_g);
            st.buf[slot0 + __popc(emit)] = r;
            if (hist) atomicAdd(hist + last_cut_g, 1ull | ((unsigned long long)(len - k + 1) << 32));
        }
        if (stopping || fin) return;
    }
}

template <int E>
__global__ void __launch_bounds__(WARPS_PER_BLOCK * 32) k_partition(const PartitionArgs a) {
    __shared__ uint64_t stages[WARPS_PER_BLOCK][STAGE];
    __shared__ uint8_t mod_w[MODW];
    if (threadIdx.x < MODW) mod_w[threadIdx.x] = (uint8_t)(threadIdx.x % a.w);
    __syncthreads();
    Stage st{stages[threadIdx.x >> 5], 0};
    // this launch's bases and fragments (the fragment table is read only inside them:
    // the entries of other pieces may not have landed yet)
    const uint64_t b0 = a.base1 ? a.base0 : 0, b1 = a.base1 ? a.base1 : a.n_bases;
    const uint64_t f_lo = a.base1 ? a.frag_lo : 0, f_hi = a.base1 ? a.frag_hi : a.n_frags;
    const uint64_t n_seg = (b1 - b0 + a.seg - 1) / a.seg;
    const uint64_t warp0 = (uint64_t)blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5);
    const uint64_t n_warps = (uint64_t)gridDim.x * WARPS_PER_BLOCK;
    for (uint64_t sgi = warp0; sgi < n_seg; sgi += n_warps) {
        const uint64_t s0 = b0 + sgi * a.seg, s1 = min(s0 + a.seg, b1);
        // last fragment starting at or before s0
        uint64_t lo = f_lo, hi = f_hi;
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (a.frag_off[mid] <= s0) lo = mid; else hi = mid;
        }
        for (uint64_t f = lo; f < f_hi; ++f) {
            const uint64_t F0 = a.frag_off[f];
            if (F0 >= s1) break;
            const uint32_t FL = a.frag_len[f];
            // a device-resident fragment table is not checked on the host: a fragment past
            // the input or too short for a (k+1)-mer is skipped and reported
            if (FL < a.k + 1 || F0 + FL > a.n_bases) {
                if ((threadIdx.x & 31) == 0) atomicOr(a.err, DERR_BAD_FRAG);
                continue;
            }
            const uint32_t M = FL - a.k + 2;
            const uint32_t j0 = s0 > F0 ? (uint32_t)(s0 - F0) : 0;
            const uint64_t e = s1 - F0;
            const uint32_t j1 = e < M ? (uint32_t)e : M;
            if (j0 < j1) sweep_fragment<E>(a, mod_w, F0, FL, j0, j1,
                                          a.hist ? a.hist + (a.frag_gbase ? a.frag_gbase[f] : 0u) : nullptr, st);
        }
    }
    stage_flush(a, st);
}

// Exclusive scan of the per-subgraph record counts (one block).
__global__ void __launch_bounds__(1024) k_bucket_scan(const unsigned long long* __restrict__ hist, uint32_t G,
                                                      uint32_t* bucket_off, uint32_t* inst, uint32_t* fill) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    const uint32_t per = (G + 1023) / 1024;
    const uint32_t b0 = t * per, b1 = min(b0 + per, G);
    uint32_t sum = 0;
    for (uint32_t b = b0; b < b1; ++b) sum += (uint32_t)hist[b];
    part[t] = sum;
    __syncthreads();
    for (uint32_t d = 1; d < 1024; d <<= 1) {
        const uint32_t v = t >= d ? part[t - d] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (uint32_t b = b0; b < b1; ++b) {
        bucket_off[b] = run;
        run += (uint32_t)hist[b];
        inst[b] = (uint32_t)(hist[b] >> 32);
        fill[b] = 0;
    }
    if (t == 1023) bucket_off[G] = part[1023];
}

// Multi-block scan for batches (millions of buckets): 8192 entries per block.
constexpr uint32_t SCAN_PER_THREAD = 8, SCAN_BLOCK = 1024, SCAN_CHUNK = SCAN_PER_THREAD * SCAN_BLOCK;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_sums, uint32_t& total) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t x = v;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= (uint32_t)d) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= (uint32_t)d) w += y;
        }
        warp_sums[lane] = w;   // inclusive
    }
    __syncthreads();
    total = warp_sums[(blockDim.x >> 5) - 1];
    const uint32_t before = wid ? warp_sums[wid - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_reduce(const unsigned long long* __restrict__ hist, uint32_t n,
                                                            uint32_t* partials) {
    __shared__ uint32_t ws[32];
    const uint64_t b0 = (uint64_t)blockIdx.x * SCAN_CHUNK + (uint64_t)threadIdx.x * SCAN_PER_THREAD;
    uint32_t sum = 0;
    for (uint32_t i = 0; i < SCAN_PER_THREAD; ++i)
        if (b0 + i < n) sum += (uint32_t)hist[b0 + i];
    uint32_t total;
    block_excl_scan(sum, ws, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_partials(uint32_t* partials, uint32_t np) {
    __shared__ uint32_t ws[32];
    const uint32_t per = (np + SCAN_BLOCK - 1) / SCAN_BLOCK;
    const uint32_t p0 = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t i = 0; i < per; ++i)
        if (p0 + i < np) sum += partials[p0 + i];
    uint32_t total;
    uint32_t run = block_excl_scan(sum, ws, total);
    for (uint32_t i = 0; i < per; ++i)
        if (p0 + i < np) { const uint32_t v = partials[p0 + i]; partials[p0 + i] = run; run += v; }
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_apply(const unsigned long long* __restrict__ hist, uint32_t n,
                                                           const uint32_t* __restrict__ partials, uint32_t* bucket_off,
                                                           uint32_t* inst, uint32_t* fill) {
    __shared__ uint32_t ws[32];
    const uint64_t b0 = (uint64_t)blockIdx.x * SCAN_CHUNK + (uint64_t)threadIdx.x * SCAN_PER_THREAD;
    unsigned long long h[SCAN_PER_THREAD];
    uint32_t sum = 0;
    for (uint32_t i = 0; i < SCAN_PER_THREAD; ++i) {
        h[i] = b0 + i < n ? hist[b0 + i] : 0ull;
        sum += (uint32_t)h[i];
    }
    uint32_t total;
    uint32_t run = partials[blockIdx.x] + block_excl_scan(sum, ws, total);
    for (uint32_t i = 0; i < SCAN_PER_THREAD; ++i) {
        if (b0 + i >= n) break;
        bucket_off[b0 + i] = run;
        inst[b0 + i] = (uint32_t)(h[i] >> 32);
        fill[b0 + i] = 0;
        run += (uint32_t)h[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) bucket_off[n] = partials[blockIdx.x] + total;
}

__global__ void k_scatter(const ScatterArgs a) {
    const uint64_t n = a.n_dev ? *a.n_dev : a.n;
    if (n > a.n) return;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = a.flat[i];
        uint32_t g = rec_g(r);
        if (a.job_pos) {   // the record's job: the last job starting at or before its first base
            const uint64_t p = rec_pos(r);
            uint32_t lo = 0, hi = a.n_jobs;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (a.job_pos[mid] <= p) lo = mid; else hi = mid;
            }
            g += lo << a.g_shift;
        }
        const uint32_t slot = atomicAdd(a.bucket_fill + g, 1u);
        a.recs[a.bucket_off[g] + slot] = r;
    }
}

}  // namespace

void launch_partition(const PartitionArgs& a, cudaStream_t s) {
    const uint64_t n_seg = ((a.base1 ? a.base1 - a.base0 : a.n_bases) + a.seg - 1) / a.seg;
    uint64_t blocks = (n_seg + WARPS_PER_BLOCK - 1) / WARPS_PER_BLOCK;
    if (blocks > (1u << 20)) blocks = 1u << 20;
    if (blocks == 0) return;
    const dim3 grid((unsigned)blocks), block(WARPS_PER_BLOCK * 32);
    switch (31 - __builtin_clz(a.w)) {   // floor(log2 w), w = k - l in [1, 126]
        case 0: k_partition<0><<<grid, block, 0, s>>>(a); break;
        case 1: k_partition<1><<<grid, block, 0, s>>>(a); break;
        case 2: k_partition<2><<<grid, block, 0, s>>>(a); break;
        case 3: k_partition<3><<<grid, block, 0, s>>>(a); break;
        case 4: k_partition<4><<<grid, block, 0, s>>>(a); break;
        case 5: k_partition<5><<<grid, block, 0, s>>>(a); break;
        default: k_partition<6><<<grid, block, 0, s>>>(a); break;
    }
}

void launch_rc_words(const uint64_t* packed, uint64_t w0, uint64_t w1, uint64_t* rcw, cudaStream_t s) {
    if (w1 <= w0) return;
    const uint64_t blocks = std::min<uint64_t>((w1 - w0 + 255) / 256, 148ull * 16);
    k_rc_words<<<(unsigned)blocks, 256, 0, s>>>(packed, w0, w1, rcw);
}

void launch_bucket_scan(const unsigned long long* hist, uint32_t G, uint32_t* bucket_off, uint32_t* inst,
                        uint32_t* fill, cudaStream_t s) {
    k_bucket_scan<<<1, 1024, 0, s>>>(hist, G, bucket_off, inst, fill);
}

void launch_bucket_scan_large(const unsigned long long* hist, uint32_t n, uint32_t* bucket_off, uint32_t* inst,
                              uint32_t* fill, uint32_t* partials, cudaStream_t s) {
    const uint32_t nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
    k_scan_reduce<<<nb, SCAN_BLOCK, 0, s>>>(hist, n, partials);
    k_scan_partials<<<1, SCAN_BLOCK, 0, s>>>(partials, nb);
    k_scan_apply<<<nb, SCAN_BLOCK, 0, s>>>(hist, n, partials, bucket_off, inst, fill);
}

void launch_scatter(const ScatterArgs& a, cudaStream_t s) {
    if (a.n == 0) return;
    uint64_t blocks = (a.n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_scatter<<<(unsigned)blocks, 256, 0, s>>>(a);
}

}  // namespace cfg
